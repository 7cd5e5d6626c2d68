"""Operator tables built on the GPU: the one-sided Jacobi SVDs of the two
pseudo-inverses and the folded C2E x M2M product run on the handle's device
(linalg_gpu.cu) with the host builder's exact arithmetic, so the tables equal
the host-built ones bit for bit (matmgnt3d_mpi.cpp:107-274 builds them lazily
per level on the host; here once per kernel and order, eagerly)."""
import time

import numpy as np
import pytest
import torch

import fmmg
import workloads as W

pytestmark = pytest.mark.gpu


def _fold_after_mixed(f, n=4000):
    """Table 6 (the folded upward operator) after one mixed evaluate formed it."""
    rng = np.random.default_rng(3)
    src = W.uniform(n, rng)
    f.setup(src, W.unit_normals(rng, n))
    den = torch.from_numpy(rng.normal(size=n * f.sd)).cuda()
    out = torch.zeros(n * f.td, dtype=torch.float64, device="cuda")
    f.evaluate_device(den, out, 1, fmmg.PREC_MIXED)
    f.sync()
    return f.operator(6)


# coefficient pairs that give the same kernel but distinct cache keys, so the
# host-only handle builds its own tables (Laplace ignores both coefficients,
# the Stokes equivalent kernel the second)
@pytest.mark.parametrize("kt,np_", [(111, 6), (111, 8), (311, 5)])
def test_device_operator_tables_bit_identical(kt, np_):
    d = fmmg.FMM3d(kt, np_=np_, pts_max=40, coefs=(1.0, 0.25), device=0)
    h = fmmg.FMM3d(kt, np_=np_, pts_max=40, coefs=(1.0, 0.2500000001), device=-1)
    for which in (0, 2):
        a, b = d.operator(which), h.operator(which)
        assert a.shape == b.shape
        assert np.array_equal(a, b), "table %d differs (max %.3e)" % (which, np.abs(a - b).max())
    fd = _fold_after_mixed(d)
    fh = h.operator(6)
    assert np.array_equal(fd, fh)


def test_navier_np8_first_handle_setup_time():
    """The Navier np = 8 operator set (two 888 x 888 SVDs, the 888 x 7104 fold)
    on the GPU: a first handle in the process builds it (coefficients no other
    test uses, so nothing is cached)."""
    t0 = time.perf_counter()
    f = fmmg.FMM3d(511, np_=8, pts_max=64, coefs=(1.0, 0.31), device=0)
    t_ops = time.perf_counter() - t0
    fold = _fold_after_mixed(f)
    t_all = time.perf_counter() - t0
    print("navier np=8 operators %.2f s, with the fold and a first mixed evaluate %.2f s" % (t_ops, t_all))
    assert np.isfinite(fold).all()
    assert t_ops < 60.0
