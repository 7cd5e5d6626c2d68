"""Mixed precision (FP32 bulk, FP64 final accumulation): accuracy against the FP64
dense sum (the reference check()) and against the plain FP64 GPU form.

Accuracy bound: relative L2 <= 1e-5 against the FP64 dense sum for Laplace
at np = 6.
"""
import numpy as np
import pytest

import fmmg
import workloads as W
from gpu_common import gpu_eval, rel_l2

pytestmark = pytest.mark.gpu


def _mixed_eval(lib, den):
    import torch
    d = torch.from_numpy(np.ascontiguousarray(den, dtype=np.float64).ravel()).cuda()
    out = torch.zeros(lib.nt * lib.td, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    lib.evaluate_device(d, out, 1, fmmg.PREC_MIXED)
    lib.sync()
    return out.cpu().numpy()


@pytest.mark.parametrize("n", [200000])
def test_mixed_laplace_np6_vs_dense(n):
    rng = np.random.default_rng(W.SEED + 2)
    src = W.sphere_clusters(n, rng)
    den = rng.normal(size=n)
    lib = fmmg.FMM3d(111, np_=6, pts_max=64)
    lib.setup(src)
    vm = _mixed_eval(lib, den)
    vd = gpu_eval(lib, den)
    idx = np.random.default_rng(1).choice(n, 4096, replace=False)
    err_m, _, dense = lib.check(den, vm, idx)
    err_d, _, _ = lib.check(den, vd, idx)
    print("mixed %.3e fp64 %.3e mixed-vs-fp64 %.3e" % (err_m, err_d, rel_l2(vm, vd)))
    assert err_m <= 1e-5
    assert rel_l2(vm, vd) <= 1e-5


@pytest.mark.parametrize("kt,np_,tol", [(121, 6, 1e-4), (321, 6, 1e-4), (511, 6, 1e-4), (312, 4, 1e-3)])
def test_mixed_other_kernels(kt, np_, tol):
    rng = np.random.default_rng(W.SEED + kt)
    n = 30000
    src = W.uniform(n, rng)
    nrm = W.unit_normals(rng, n)
    lib = fmmg.FMM3d(kt, np_=np_, pts_max=64)
    lib.setup(src, nrm)
    den = rng.normal(size=n * lib.sd)
    vm = _mixed_eval(lib, den)
    vd = gpu_eval(lib, den)
    assert rel_l2(vm, vd) <= tol


@pytest.mark.parametrize("kt", [321, 121])
def test_mixed_double_layer_on_dense_surfaces(kt):
    """Double-layer kernels on 1,048,576 points on 64 ellipsoids (the Stokes
    double-layer workload's geometry): near-coincident pairs on a smooth
    surface have n.(x - y) = O(r^2), which FP32 offsets or normals cannot
    resolve; the near field forms it in FP64.  Per right-hand side the mixed
    form stays within 5e-6 of the FP64 form (the FP64 form itself is at the
    np = 6 truncation error, ~4e-5 against the dense sum for Stokes)."""
    import torch
    cfg = W.config3(k_rhs=2)
    src, nrm = cfg["src"], cfg["nrm"]
    n = src.shape[0]
    lib = fmmg.FMM3d(kt, np_=6, pts_max=64)
    lib.setup(src, nrm)
    rng = np.random.default_rng(kt)
    den = rng.normal(size=(2, n * lib.sd))
    d = torch.from_numpy(den).cuda()
    om = torch.zeros(2, n * lib.td, dtype=torch.float64, device="cuda")
    od = torch.zeros_like(om)
    torch.cuda.synchronize()
    lib.evaluate_device(d, om, 2, fmmg.PREC_MIXED)
    lib.evaluate_device(d, od, 2, fmmg.PREC_FP64)
    lib.sync()
    vm, vd = om.cpu().numpy(), od.cpu().numpy()
    for r in range(2):
        e = rel_l2(vm[r], vd[r])
        print("kernel %d rhs %d mixed-vs-fp64 %.3e" % (kt, r, e))
        assert e <= 5e-6


def test_mixed_host_path_and_stage_masks():
    rng = np.random.default_rng(4)
    n = 20000
    src = W.uniform(n, rng)
    den = rng.normal(size=n)
    lib = fmmg.FMM3d(111, np_=4, pts_max=40)
    lib.setup(src)
    lib.set_precision(fmmg.PREC_MIXED)
    vh = lib.evaluate(den).ravel()
    vm = _mixed_eval(lib, den)
    assert rel_l2(vh, vm) <= 1e-12  # same arithmetic through the host-buffer call
    vd = gpu_eval(lib, den)
    assert rel_l2(vm, vd) <= 1e-5


def test_mixed_multi_rhs_matches_single_rhs():
    import torch
    rng = np.random.default_rng(8)
    n = 30000
    src = W.sphere_clusters(n, rng)
    lib = fmmg.FMM3d(111, np_=6, pts_max=64)
    lib.setup(src)
    k = 11  # exercises blocks of 8, 2 and 1 right-hand sides
    D = rng.normal(size=(k, n))
    d = torch.from_numpy(D).cuda()
    out = torch.zeros(k, n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    lib.evaluate_device(d, out, k, fmmg.PREC_MIXED)
    lib.sync()
    V = out.cpu().numpy()
    # The batched and single forms may split the K sums of the FP32 row GEMMs
    # differently (split-K is chosen by problem size), so they agree to FP32
    # rounding; a right-hand side mixed up with another would differ by O(1).
    for r in (0, 7, 10):
        assert rel_l2(V[r], _mixed_eval(lib, D[r])) <= 1e-6
    nrm = W.unit_normals(rng, n)
    g = fmmg.FMM3d(321, np_=4, pts_max=64)
    g.setup(src, nrm)
    D3 = rng.normal(size=(5, 3 * n))
    out3 = torch.zeros(5, 3 * n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    g.evaluate_device(torch.from_numpy(D3).cuda(), out3, 5, fmmg.PREC_MIXED)
    g.sync()
    V3 = out3.cpu().numpy()
    for r in (0, 4):
        assert rel_l2(V3[r], _mixed_eval(g, D3[r])) <= 1e-6


@pytest.mark.parametrize("k", [1, 8])
def test_gemm_paths_agree(k):
    """The three kernels of the FP32 row GEMMs on one evaluate: the tensor
    cores (3xTF32, tcgen05, the default), the 128 x 160 CUDA-core tiles and
    the 128 x 64 CUDA-core tiles.  The CUDA-core kernels differ only in
    summation order (split K, where the uniform X scale is applied); 3xTF32
    represents each operand to 2^-22 and drops the lo*lo term, with every
    32-wide K block summed in FP32 (~1e-6 from the others at np = 6).  All
    meet the 1e-5 bound against the dense FP64 sum, the accuracy gate of the
    mixed form."""
    import torch
    rng = np.random.default_rng(41 + k)
    n = 60000
    src = W.sphere_clusters(n, rng)
    lib = fmmg.FMM3d(111, np_=6, pts_max=64)
    lib.setup(src)
    D = rng.normal(size=(k, n))
    outs = {}
    for path in ("tc", "narrow", "wide"):
        lib.set_gemm_path(path)
        out = torch.zeros(k, n, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        lib.evaluate_device(torch.from_numpy(D).cuda(), out, k, fmmg.PREC_MIXED)
        lib.sync()
        assert lib.device_error() == 0
        outs[path] = out.cpu().numpy()
    print("k %d wide vs narrow %.3e, wide vs tc %.3e" % (
        k, rel_l2(outs["wide"], outs["narrow"]), rel_l2(outs["wide"], outs["tc"])))
    assert rel_l2(outs["wide"], outs["narrow"]) <= 1e-6
    assert rel_l2(outs["tc"], outs["wide"]) <= 5e-6
    idx = rng.choice(n, 2000, replace=False)
    for r in (0, k - 1):
        for path in outs:
            rel, _, _ = lib.check(D[r], outs[path][r], idx)
            print("k %d rhs %d %s rel err vs dense %.3e" % (k, r, path, rel))
            assert rel <= 1e-5
    with pytest.raises(ValueError):
        lib.set_gemm_path("fast")


@pytest.mark.parametrize("np_", [3, 4, 5, 8])
def test_mixed_rhs_blocks_at_other_np(np_):
    """The 8-right-hand-side transforms and Hadamard at every grid size they
    are instantiated for: a block of 3 equals 3 single evaluations to FP32
    rounding (split-K may sum the GEMMs in another order)."""
    import torch
    rng = np.random.default_rng(50 + np_)
    n = 30000
    src = W.sphere_clusters(n, rng)
    lib = fmmg.FMM3d(111, np_=np_, pts_max=64)
    lib.setup(src)
    k = 3
    D = rng.normal(size=(k, n))
    out = torch.zeros(k, n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    lib.evaluate_device(torch.from_numpy(D).cuda(), out, k, fmmg.PREC_MIXED)
    lib.sync()
    V = out.cpu().numpy()
    for r in range(k):
        assert rel_l2(V[r], _mixed_eval(lib, D[r])) <= 1e-6


@pytest.mark.parametrize("k", [5, 8, 12])
def test_hadamard_forms(k):
    """The four forms of the FP32 Hadamard on one evaluate.  Forms 1 and 2
    (27 product accumulators, one or two right-hand sides per thread) do, per
    right-hand side, the same operations in the same order, and so do forms 3
    and 4 (8 output-child accumulators, two or four right-hand sides per
    thread): each pair agrees bit for bit (odd k leaves lanes with unused
    right-hand sides, k = 12 spans two blocks of 8).  Between the pairs only
    the order of the sums differs."""
    import torch
    rng = np.random.default_rng(77 + k)
    n = 40000
    src = W.sphere_clusters(n, rng)
    lib = fmmg.FMM3d(111, np_=6, pts_max=64)
    lib.setup(src)
    D = torch.from_numpy(rng.normal(size=(k, n))).cuda()
    outs = {}
    for form in (1, 2, 3, 4):
        assert lib.tuning({"had_fp32_rhs_per_thread": form})["had_fp32_rhs_per_thread"] == form
        out = torch.zeros(k, n, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        lib.evaluate_device(D, out, k, fmmg.PREC_MIXED)
        lib.sync()
        assert lib.device_error() == 0
        outs[form] = out.cpu().numpy()
    assert np.array_equal(outs[1], outs[2])
    assert np.array_equal(outs[3], outs[4])
    assert rel_l2(outs[4], outs[1]) <= 1e-6
    with pytest.raises(fmmg.FmmgError):
        lib.tuning({"had_fp32_rhs_per_thread": 5})


def test_mixed_follows_replaced_pinv():
    """fmmg_operator(set) replaces the pseudo-inverses: the FP32 pass refactors
    each from its explicit table (SVD) and rebuilds the folded C2E x M2M
    product, so the mixed form still matches the FP64 form on the replaced
    operator set."""
    import torch
    rng = np.random.default_rng(91)
    n = 30000
    src = W.sphere_clusters(n, rng)
    f = fmmg.FMM3d(111, np_=6, pts_max=64)
    f.setup(src)
    D = torch.from_numpy(rng.normal(size=(2, n))).cuda()

    def both():
        outs = []
        for prec in (fmmg.PREC_FP64, fmmg.PREC_MIXED):
            out = torch.zeros(2, n, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            f.evaluate_device(D, out, 2, prec)
            f.sync()
            outs.append(out.cpu().numpy())
        return outs

    d0, m0 = both()
    assert rel_l2(m0, d0) <= 1e-5
    for which in (0, 2):
        f.set_operator(which, 0, 0.5 * f.operator(which))
    d1, m1 = both()
    print("replaced pinv: fp64 change %.3e, mixed vs fp64 %.3e" % (rel_l2(d1, d0), rel_l2(m1, d1)))
    assert rel_l2(d1, d0) > 1e-2  # the replacement is visible
    assert rel_l2(m1, d1) <= 1e-5


@pytest.mark.parametrize("np_", [5, 6])
def test_mixed_follows_replaced_translation_spectra(np_):
    """The FP32 pass transforms on the (2np-1)^3 grid, the reference's tables
    live on the (2np)^3 grid: a translation spectrum the caller replaces is
    converted exactly (inverse r2c to the kernel samples, the offsets
    -(np-1)..np-1 the band-to-band convolution reads, r2c on the odd grid), so
    the mixed form still matches the FP64 form.  Two translations are swapped,
    which changes the V list visibly."""
    import torch
    rng = np.random.default_rng(92 + np_)
    n = 30000
    src = W.sphere_clusters(n, rng)
    f = fmmg.FMM3d(111, np_=np_, pts_max=64)
    f.setup(src)
    D = torch.from_numpy(rng.normal(size=(2, n))).cuda()

    def both():
        outs = []
        for prec in (fmmg.PREC_FP64, fmmg.PREC_MIXED):
            out = torch.zeros(2, n, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            f.evaluate_device(D, out, 2, prec)
            f.sync()
            outs.append(out.cpu().numpy())
        return outs

    d0, m0 = both()
    assert rel_l2(m0, d0) <= 1e-5
    a, b = f.operator(4, 0), f.operator(4, 315)
    f.set_operator(4, 0, b)
    f.set_operator(4, 315, a)
    d1, m1 = both()
    print("np %d swapped spectra: fp64 change %.3e, mixed vs fp64 %.3e" % (np_, rel_l2(d1, d0), rel_l2(m1, d1)))
    assert rel_l2(d1, d0) > 1e-4
    assert rel_l2(m1, d1) <= 1e-5


@pytest.mark.parametrize("np_", [3, 4, 5, 6, 7, 8])
def test_mixed_matches_fp64_form_every_np(np_):
    """The mixed form transforms on the (2np-1)^3 grid, the FP64 form on the
    reference's (2np)^3 grid: for every order both compute the same operator,
    so they agree to the FP32 rounding of the mixed form (k = 1 and a block of
    8 right-hand sides)."""
    import torch
    rng = np.random.default_rng(60 + np_)
    n = 30000
    src = W.sphere_clusters(n, rng)
    lib = fmmg.FMM3d(111, np_=np_, pts_max=64)
    lib.setup(src)
    for k in (1, 8):
        D = torch.from_numpy(rng.normal(size=(k, n))).cuda()
        outs = []
        for prec in (fmmg.PREC_FP64, fmmg.PREC_MIXED):
            out = torch.zeros(k, n, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            lib.evaluate_device(D, out, k, prec)
            lib.sync()
            outs.append(out.cpu().numpy())
        err = rel_l2(outs[1], outs[0])
        print("np %d k %d mixed vs fp64 %.3e" % (np_, k, err))
        assert err <= 2e-5


def test_mixed_form_after_a_second_setup():
    """A handle set up again on moved points (its device arrays, the
    tensor-core operator copies among them, freed and rebuilt) evaluates the
    mixed form exactly like a fresh handle on those points."""
    import torch
    rng = np.random.default_rng(61)
    n, k = 30000, 8
    a = W.sphere_clusters(n, rng)
    b = np.clip(a + 0.01 * rng.normal(size=a.shape), 0.0, 1.0 - 1e-12)
    D = torch.from_numpy(rng.normal(size=(k, n))).cuda()

    def ev(lib):
        out = torch.zeros(k, n, dtype=torch.float64, device="cuda")
        lib.evaluate_device(D, out, k, fmmg.PREC_MIXED)
        lib.sync()
        assert lib.device_error() == 0
        return out.cpu().numpy()

    lib = fmmg.FMM3d(111, np_=6, pts_max=64)
    lib.setup(a)
    ev(lib)
    lib.setup(b)
    again = ev(lib)
    fresh = fmmg.FMM3d(111, np_=6, pts_max=64)
    fresh.setup(b)
    assert np.array_equal(again, ev(fresh))


def test_headline_workload_every_rhs_within_budget():
    """The 1,048,576-point benchmark workload in the mixed form with 8 random
    N(0, 1) right-hand sides: every one of them within the 1e-5 budget against
    the FP64 dense sum at 4,096 sampled targets.  (Near-coincident points of
    the Gaussian clusters once made single right-hand sides reach 5e-5: their
    near-field offsets now keep the separation to FP32 precision.)"""
    import torch
    cfg = W.config2(1 << 20)
    n, k = 1 << 20, 8
    lib = fmmg.FMM3d(111, np_=6, pts_max=64)
    lib.setup(cfg["src"])
    D = np.random.default_rng(5).normal(size=(k, n))
    out = torch.zeros(k, n, dtype=torch.float64, device="cuda")
    lib.evaluate_device(torch.from_numpy(D).cuda(), out, k, fmmg.PREC_MIXED)
    lib.sync()
    assert lib.device_error() == 0
    V = out.cpu().numpy()
    idx = np.random.default_rng(99).choice(n, 4096, replace=False)
    errs = [lib.check(D[r], V[r], idx)[0] for r in range(k)]
    print("1M mixed k=8 per-rhs rel err vs dense: %s" % ["%.2e" % e for e in errs])
    assert max(errs) <= 1e-5
