"""The oracle pinned against the reference's own code.

oracle/_ref holds the reference's kernel3d_mpi.cpp, matmgnt3d_mpi.cpp,
vecmatop.cpp and svdrep.cpp compiled unchanged (oracle/ref/Makefile), with
stand-in PETSc/FFTW headers, the netlib BLAS algorithms and FFTW's r2c/c2r
semantics restated, and scipy's LAPACK dgesvd (oracle/ref_code.py).  Against
it:

* the kernel blocks of all 8 setup() kernels and the 3 equivalent kernels,
  and the surface and regular grids, are bit-identical;
* the M2M and L2L tables (pure kernel evaluations) are bit-identical;
* the translation spectra and one whole V-list interaction (embed, r2c,
  Hadamard, c2r, gather) agree to DFT rounding (two DFT restatements);
* the C2E pseudo-inverses come from different SVD codes (LAPACK dgesvd here,
  a one-sided Jacobi in the oracle and the library): they agree where the
  operator acts (on the range of the check map) and the whole evaluate run
  on the reference-built tables stays within a few times the reference
  arithmetic's own reordering floor.

Skipped where the reference tree was not there to build the library.
"""
import numpy as np
import pytest

import oracle as O

R = pytest.importorskip("ref_code")
if not R.available():
    pytest.skip("the reference's code is not built here", allow_module_level=True)

KERNELS = (111, 121, 311, 312, 321, 322, 511, 521)
EQUIV = {111: 111, 121: 111, 311: 301, 312: 301, 321: 301, 322: 301, 511: 511, 521: 511}


def _pts(rng, n):
    return rng.random((n, 3))


@pytest.mark.parametrize("kt", KERNELS + (301,))
def test_kernel_blocks_bit_identical(kt):
    rng = np.random.default_rng(kt)
    src = _pts(rng, 40)
    nrm = rng.normal(size=(40, 3))
    trg = np.concatenate([_pts(rng, 25), src[:3], src[3:5] + 1e-9])  # coincident and r < 1e-8 pairs
    for coefs in ((1.0, 0.25), (0.7, 0.3)):
        a = R.kernel_matrix(kt, src, nrm, trg, coefs)
        b = O.kernel_matrix(kt, src, nrm, trg, coefs)
        assert np.array_equal(a, b)


@pytest.mark.parametrize("np_", [3, 4, 5, 6, 7, 8])
def test_surfaces_and_regular_grid_bit_identical(np_):
    for radius in (1.0, 3.0):
        assert np.array_equal(R.sampos(np_, radius), O.sampos(np_, radius))
        assert np.array_equal(R.regpos(np_, radius), O.regpos(np_, radius))
    assert np.array_equal(R.sampos(np_ + 2, 3.0), O.sampos(np_ + 2, 3.0))


@pytest.mark.parametrize("kt,np_", [(111, 4), (111, 6), (321, 4), (511, 5), (121, 8)])
def test_operator_tables(kt, np_):
    mm = EQUIV[kt]
    o = O.Oracle(kt, np_=np_)
    for which in (1, 3):  # M2M and L2L: kernel evaluations only
        for i in range(8):
            assert np.array_equal(R.operator(mm, np_, which, i), o.operator(which, i)), (which, i)
    for i in (0, 57, 158, 315):  # translation spectra: two DFT restatements
        a, b = R.operator(mm, np_, 4, i), o.operator(4, i)
        assert np.linalg.norm(a - b) <= 2e-15 * np.linalg.norm(a), i
    # pseudo-inverses from different SVD codes: equal where they act, P K = P' K
    s = o.sizes()
    sd, td = O.src_dof(mm), O.trg_dof(mm)
    for which, chk, den in ((0, O.sampos(np_ + 2, 3.0), O.sampos(np_, 1.0)), (2, O.sampos(np_, 1.0),
                                                                              O.sampos(np_, 3.0))):
        K = O.kernel_matrix(mm, den, den, chk)
        P_ref = R.operator(mm, np_, which).reshape(K.shape[0], K.shape[1]).T  # column-major n x m
        P_orc = o.operator(which).reshape(K.shape[0], K.shape[1]).T
        assert P_ref.shape == (len(den) * sd, len(chk) * td) == (s["UE" if which == 0 else "DE"] * sd, K.shape[0])
        # both sides of K P K carry the rounding of a product through P, whose
        # norm is the inverse cutoff 10^(np+1): eps_mach x 10^(np+1)
        proj_ref, proj_orc = K @ P_ref @ K, K @ P_orc @ K
        assert np.linalg.norm(proj_ref - proj_orc) <= 2.2e-16 * 10.0 ** (np_ + 1) * np.linalg.norm(K), which
        # and both reproduce K up to the truncated singular values
        assert np.linalg.norm(proj_ref - K) <= 10.0 ** (-np_ + 1) * np.linalg.norm(K), which


@pytest.mark.parametrize("kt,np_", [(111, 4), (111, 6), (111, 8), (321, 6), (511, 6)])
def test_one_v_list_interaction(kt, np_):
    mm = EQUIV[kt]
    o = O.Oracle(kt, np_=np_)
    rng = np.random.default_rng(np_ + kt)
    den = rng.normal(size=o.sizes()["UE"] * O.src_dof(mm))
    for level, tid in ((0, 0), (2, 31), (4, 200), (7, 315)):
        a = R.m2l(mm, np_, level, tid, den)
        b = o.m2l_single(level, tid, den)
        assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(a), (level, tid)


@pytest.mark.parametrize("kt,np_", [(111, 4), (111, 6), (121, 6), (321, 6), (511, 6), (111, 8)])
def test_evaluate_on_reference_built_tables(kt, np_):
    """The oracle's evaluate on the operator tables the reference's own
    MatMgnt3d_MPI builds (LAPACK pseudo-inverses) against the oracle on its
    own tables: within 4x the reordering floor of the reference arithmetic
    (the oracle against itself with every operator GEMV summed in reverse),
    and within 1e-10 up to np = 6."""
    mm = EQUIV[kt]
    rng = np.random.default_rng(31 + np_)
    n = 5000
    m = n // 2
    v = rng.normal(size=(m, 3))
    src = np.concatenate([0.5 + 0.45 * v / np.linalg.norm(v, axis=1)[:, None], rng.random((n - m, 3))])
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1)[:, None]
    o = O.Oracle(kt, np_=np_, pts_max=40, nthreads=8)
    o.setup(src, nrm, src)
    den = rng.uniform(-1, 1, n * O.src_dof(kt))
    own = o.evaluate(den)
    o.set_gemv_order(True)
    floor = np.linalg.norm(o.evaluate(den) - own) / np.linalg.norm(own)
    o.set_gemv_order(False)
    for which, idxs in ((0, [0]), (1, range(8)), (2, [0]), (3, range(8)), (4, range(316))):
        for i in idxs:
            o.set_operator(which, i, R.operator(mm, np_, which, i))
    err = np.linalg.norm(o.evaluate(den) - own) / np.linalg.norm(own)
    assert err <= max(1e-10 if np_ <= 6 else 0.0, 4.0 * floor), (err, floor)
