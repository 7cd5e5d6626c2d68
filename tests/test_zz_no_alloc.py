"""fmmg_dense_noalloc: the dense direct sum for callers that cannot allocate.

Callers that record work into a CUDA graph, run inside a memory pool that
forbids driver allocations, or sit on a latency-critical path cannot call
cudaMalloc when they need a result; this entry point keeps its only scratch (the
accumulation buffer) in a fixed array inside the library.  Its output must match
the dense sums of the existing allocating entry point, fmmg_check(), to FP64
rounding (the two sum the same terms; atomics make the order differ), on two
calls in a row (the second call reuses the array the first one left behind).
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import fmmg

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative L2, FP64 sums of the same terms in a different order


def _noalloc(kt, src, nrm, den, trg, coefs=(1.0, 0.25)):
    import torch
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    ds, dn, dd, dt = d(src), d(nrm), d(den), d(trg)
    td = fmmg.KERNELS.get(kt, (1, 1))[1]
    out = torch.full((trg.shape[0] * td,), np.nan, dtype=torch.float64, device="cuda")
    cf = np.ascontiguousarray(coefs, dtype=np.float64)
    torch.cuda.synchronize()
    st = fmmg.lib().fmmg_dense_noalloc(kt, cf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), src.shape[0],
                                       ds.data_ptr(), dn.data_ptr(), dd.data_ptr(), trg.shape[0], dt.data_ptr(),
                                       out.data_ptr(), None)
    torch.cuda.synchronize()
    return st, out.cpu().numpy()


@pytest.mark.parametrize("kt", [111, 121, 321])
def test_noalloc_matches_check_dense_sums_twice(kt):
    rng = np.random.default_rng(77 + kt)
    n = 20000
    src = rng.random((n, 3))
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1)[:, None]
    f = fmmg.FMM3d(kt, np_=4, pts_max=64)
    f.setup(src, nrm)
    for call in range(2):
        den = rng.normal(size=n * f.sd)
        idx = rng.choice(n, 3000, replace=False)
        val = f.evaluate(den)
        _, _, dense = f.check(den, val, idx)  # the allocating entry point
        st, got = _noalloc(kt, src, nrm, den, src[idx])
        assert st == fmmg.FMMG_OK
        ref = dense.ravel()
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= TOL, call


@pytest.mark.parametrize("kt", [111, 121, 321])
def test_noalloc_matches_the_oracle_dense_sum(kt):
    """An independent check of the kernel formulas and the normal indexing:
    the CPU oracle's FP64 dense sum (the reference check()'s Dense3d sum) at a
    few hundred targets, on two calls in a row."""
    import oracle as O
    rng = np.random.default_rng(5 + kt)
    n = 6000
    src = rng.random((n, 3))
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1)[:, None]
    sd = O.src_dof(kt)
    for call in range(2):
        den = rng.normal(size=n * sd)
        trg = rng.random((300, 3))
        st, got = _noalloc(kt, src, nrm, den, trg)
        assert st == fmmg.FMMG_OK
        ref = O.dense(kt, src, nrm, den, trg)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= TOL, call


def test_noalloc_zero_targets_and_navier_nu_one():
    rng = np.random.default_rng(4)
    src = rng.random((10, 3))
    # no targets: nothing to sum, like fmmg_setup with zero targets
    import torch
    ds = torch.from_numpy(src).cuda()
    dd = torch.from_numpy(rng.normal(size=10)).cuda()
    st = fmmg.lib().fmmg_dense_noalloc(111, None, 10, ds.data_ptr(), None, dd.data_ptr(), 0, None, None, None)
    torch.cuda.synchronize()
    assert st == fmmg.FMMG_OK
    # the Navier kernels divide by 1 - nu: refused as fmmg_create refuses them
    st, _ = _noalloc(511, src, src, rng.normal(size=30), src, coefs=(1.0, 1.0))
    assert st == fmmg.FMMG_INVALID_ARG


def test_noalloc_rejects_sizes_beyond_the_fixed_scratch():
    rng = np.random.default_rng(3)
    src = rng.random((10, 3))
    trg = rng.random(((1 << 20) // 3 + 1, 3))  # 3 values per target: one more than fits
    st, _ = _noalloc(321, src, src, rng.normal(size=30), trg)
    assert st == fmmg.FMMG_INVALID_ARG
    st, _ = _noalloc(999, src, src, rng.normal(size=10), src)
    assert st == fmmg.FMMG_NOT_SUPPORTED
