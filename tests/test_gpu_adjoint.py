"""The hand-written adjoint: transposed FMM (d/d density) and target-position gradient.

The adjoint runs every forward stage transposed, in reverse order, on the same
tree and operators, so it must equal the transpose of the forward FMM operator
to FP64 rounding -- checked against the operator the oracle evaluates
(explicit matrix on small cases, bilinear identity on large ones).  Against
the exact (dense) transposed sums it carries the FMM's own approximation error.
The target-position gradient is the exact gradient of the FMM approximant, so
it matches central differences of the evaluator itself closely.
"""
import numpy as np
import pytest

import fmmg
import oracle as O
from gpu_common import SEED, gpu_eval, points, rel_l2, share_operators, unit_normals

pytestmark = pytest.mark.gpu

EXACT = 1e-10  # the adjoint vs the transpose of the same FMM operator (FP64)
KERNELS = (111, 121, 311, 312, 321, 322, 511, 521)


def _setup(kt, n, np_=4, pts=6, kind="sphere_clusters", seed=1, n_trg=None):
    rng = np.random.default_rng(SEED + seed)
    src = points(kind, n, rng)
    nrm = unit_normals(rng, n)
    trg = src if n_trg is None else rng.random((n_trg, 3))
    f = fmmg.FMM3d(kt, np_=np_, pts_max=pts)
    f.setup(src, nrm, trg)
    return f, src, nrm, trg, rng


def _gpu_matrix(f):
    """The forward FMM operator, column by column (k right-hand sides at once)."""
    import torch
    m = f.ns * f.sd
    den = torch.eye(m, dtype=torch.float64, device="cuda").contiguous()
    out = torch.zeros((m, f.nt * f.td), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    f.evaluate_device(den, out, k=m)
    f.sync()
    return out.cpu().numpy().T  # [nt*td, ns*sd]


@pytest.mark.parametrize("kt", KERNELS)
def test_adjoint_is_transpose_of_forward_operator(kt):
    n = 300 if fmmg.KERNELS[kt][0] == 1 else 160
    f, *_, rng = _setup(kt, n, pts=5)
    s = f.plan_stats()
    assert s["v_interactions"] > 0 and s["m2t_pairs"] > 0 and s["s2l_pairs"] > 0  # every list is exercised
    A = _gpu_matrix(f)
    for _ in range(2):
        w = rng.normal(size=f.nt * f.td)
        g, _ = f.adjoint(w)
        assert rel_l2(g.ravel(), A.T @ w) <= EXACT


@pytest.mark.parametrize("kt", [111, 121])
def test_adjoint_matches_oracle_operator(kt):
    """Pinned to the oracle: A^T w with A the oracle's own FMM matrix (shared operators)."""
    rng = np.random.default_rng(SEED + 5)
    n = 150
    src = points("sphere_clusters", n, rng)
    nrm = unit_normals(rng, n)
    f = fmmg.FMM3d(kt, np_=4, pts_max=4)
    f.setup(src, nrm)
    orc = O.Oracle(kt, np_=4, pts_max=4)
    orc.setup(src, nrm, src)
    share_operators(f, orc)
    A = np.stack([orc.evaluate(np.eye(n)[j]).ravel() for j in range(n)], 1)
    w = rng.normal(size=n)
    g, _ = f.adjoint(w)
    assert rel_l2(g.ravel(), A.T @ w) <= EXACT


@pytest.mark.parametrize("kt,n,np_", [(111, 200000, 6), (121, 60000, 6), (321, 40000, 5), (511, 30000, 4)])
def test_adjoint_bilinear_identity_large(kt, n, np_):
    """<A sigma, w> = <sigma, A^T w> at sizes where the matrix cannot be formed."""
    f, *_, rng = _setup(kt, n, np_=np_, pts=64, seed=11)
    sig = rng.normal(size=n * f.sd)
    w = rng.normal(size=f.nt * f.td)
    phi = gpu_eval(f, sig)
    g, _ = f.adjoint(w)
    lhs, rhs = float(phi.ravel() @ w), float(sig @ g.ravel())
    assert abs(lhs - rhs) <= 1e-12 * np.linalg.norm(phi) * np.linalg.norm(w)


def _dense_transpose(kt, src, nrm, trg, w, idx, coefs=(1.0, 0.25)):
    """g[s] = sum_t K(x_t - y_s; n_s)^T w_t for sources idx (oracle kernel blocks)."""
    sd, td = fmmg.KERNELS[kt]
    out = np.zeros((len(idx), sd))
    W = w.reshape(-1, td)
    for a, s in enumerate(idx):
        K = O.kernel_matrix(kt, src[s:s + 1], nrm[s:s + 1], trg, coefs)  # [nt*td, sd]
        out[a] = K.T @ W.ravel()
    return out


@pytest.mark.parametrize("kt", [111, 121, 321])
def test_adjoint_vs_dense_transposed_sums(kt):
    n = 20000
    f, src, nrm, trg, rng = _setup(kt, n, np_=6, pts=64, seed=3)
    w = rng.normal(size=f.nt * f.td)
    g, _ = f.adjoint(w)
    idx = rng.choice(n, 300, replace=False)
    ref = _dense_transpose(kt, src, nrm, trg, w, idx)
    tol = 1e-5 if kt != 321 else 1e-4
    assert rel_l2(g[idx], ref) <= tol


def _grad_dense(kt, src, nrm, den, trg, w, idx):
    """w_t * grad_x sum_s K(x - y_s; n_s) den_s at targets idx."""
    C = 1.0 / (4 * np.pi)
    out = np.zeros((len(idx), 3))
    for a, t in enumerate(idx):
        d = trg[t] - src
        r2 = (d * d).sum(1)
        ok = r2 >= 1e-16
        d, r2, dn, nn = d[ok], r2[ok], den[ok], nrm[ok]
        ir3 = r2 ** -1.5
        if kt == 111:
            G = -C * ir3[:, None] * d
        else:
            rn = (d * nn).sum(1)
            G = -C * (nn * ir3[:, None] - 3.0 * (rn * r2 ** -2.5)[:, None] * d)
        out[a] = w[t] * (G * dn[:, None]).sum(0)
    return out


@pytest.mark.parametrize("kt", [111, 121])
def test_target_gradient_vs_dense(kt):
    n = 20000
    f, src, nrm, trg, rng = _setup(kt, n, np_=6, pts=64, seed=4, n_trg=5000)
    den = rng.normal(size=n)
    w = rng.normal(size=f.nt)
    _, gt = f.adjoint(w, den, target_grad=True)
    idx = rng.choice(f.nt, 200, replace=False)
    ref = _grad_dense(kt, src, nrm, den, trg, w, idx)
    assert rel_l2(gt[idx], ref) <= 1e-4


@pytest.mark.parametrize("kt", [111, 121])
def test_target_gradient_central_differences(kt):
    """The gradient of the FMM approximant itself: a target moved by +-h stays
    in its leaf, so differences of evaluate() converge to it.  Targets near a
    clustered source have large third derivatives (|grad| ~ 1e3 at distance
    ~7e-3 gives an O(h^2) central-difference error ~4e-3 at h = 1e-5), so the
    central differences are Richardson-extrapolated (error O(h^4))."""
    n, h = 20000, 1e-5
    f, src, nrm, trg, rng = _setup(kt, n, np_=6, pts=64, seed=6, n_trg=2000)
    den = rng.normal(size=n)
    w = rng.normal(size=f.nt)
    _, gt = f.adjoint(w, den, target_grad=True)

    def central(t, d, step):
        vals = []
        for sgn in (1, -1):
            moved = trg.copy()
            moved[t, d] += sgn * step
            g2 = fmmg.FMM3d(kt, np_=6, pts_max=64)
            g2.setup(src, nrm, moved)
            vals.append(g2.evaluate(den)[t, 0])
            g2.close()
        return w[t] * (vals[0] - vals[1]) / (2 * step)

    for t in rng.choice(f.nt, 3, replace=False):
        fd = np.array([(4 * central(t, d, h / 2) - central(t, d, h)) / 3 for d in range(3)])
        assert np.linalg.norm(fd - gt[t]) <= 1e-6 * np.linalg.norm(gt[t]) + 1e-9


def test_torch_autograd_function():
    import torch
    import fmmg_torch
    n = 30000
    f, src, nrm, trg, rng = _setup(111, n, np_=6, pts=64, seed=8, n_trg=4000)
    den = torch.tensor(rng.normal(size=(n, 1)), dtype=torch.float64, device="cuda", requires_grad=True)
    x = torch.tensor(trg, dtype=torch.float64, device="cuda", requires_grad=True)
    wt = torch.tensor(rng.normal(size=(f.nt, 1)), dtype=torch.float64, device="cuda")
    phi = fmmg_torch.fmm_apply(f, den, x)
    loss = (phi * wt).sum()
    loss.backward()
    g, gt = f.adjoint(wt.cpu().numpy().ravel(), den.detach().cpu().numpy().ravel(), target_grad=True)
    assert den.grad.shape == den.shape and x.grad.shape == x.shape
    assert rel_l2(den.grad.cpu().numpy(), g) <= 1e-14
    assert rel_l2(x.grad.cpu().numpy(), gt) <= 1e-14
    ref = gpu_eval(f, den.detach().cpu().numpy())
    assert rel_l2(phi.detach().cpu().numpy(), ref) <= 1e-14


def test_adjoint_edge_cases():
    rng = np.random.default_rng(SEED + 9)
    src = rng.random((500, 3))
    f = fmmg.FMM3d(111, np_=4, pts_max=20)
    f.setup(src, None, np.zeros((0, 3)))  # no targets: A^T w = 0
    g, _ = f.adjoint(np.zeros(0))
    assert np.all(g == 0)
    f2 = fmmg.FMM3d(311, np_=4, pts_max=20)
    f2.setup(src)
    with pytest.raises(fmmg.FmmgError) as e:
        f2.adjoint(np.zeros(1500), np.zeros(1500), target_grad=True)
    assert e.value.status == fmmg.FMMG_NOT_SUPPORTED


def test_adjoint_k_right_hand_sides():
    """k right-hand sides in one call equal k single calls (same arithmetic)."""
    f, src, nrm, trg, rng = _setup(111, 20000, np_=6, pts=64, seed=12, n_trg=3000)
    k = 3
    w = rng.normal(size=(k, f.nt))
    den = rng.normal(size=(k, f.ns))
    g, gt = f.adjoint(w, den, target_grad=True, k=k)
    assert g.shape == (k, f.ns, 1) and gt.shape == (k, f.nt, 3)
    for r in range(k):
        g1, gt1 = f.adjoint(w[r], den[r], target_grad=True)
        assert np.array_equal(g[r], g1) and np.array_equal(gt[r], gt1)


@pytest.mark.parametrize("precision", [fmmg.PREC_FP64, fmmg.PREC_MIXED])
def test_torch_autograd_k_right_hand_sides(precision):
    """fmm_apply on a [k, n_src, 1] block: the forward equals the evaluate of
    the block in the given precision, the density gradient is the transposed
    FMM of each right-hand side, and the target gradient their sum."""
    import torch
    import fmmg_torch
    n, k = 30000, 4
    f, src, nrm, trg, rng = _setup(111, n, np_=6, pts=64, seed=14, n_trg=4000)
    den = torch.tensor(rng.normal(size=(k, n, 1)), dtype=torch.float64, device="cuda", requires_grad=True)
    x = torch.tensor(trg, dtype=torch.float64, device="cuda", requires_grad=True)
    wt = torch.tensor(rng.normal(size=(k, f.nt, 1)), dtype=torch.float64, device="cuda")
    phi = fmmg_torch.fmm_apply(f, den, x, precision)
    assert phi.shape == (k, f.nt, 1)
    (phi * wt).sum().backward()
    ref = torch.zeros(k, f.nt, dtype=torch.float64, device="cuda")
    f.evaluate_device(den.detach().view(k, n).contiguous(), ref, k, precision)
    f.sync()
    assert torch.equal(phi.detach().view(k, f.nt), ref)
    g, gt = f.adjoint(wt.cpu().numpy().reshape(k, -1), den.detach().cpu().numpy().reshape(k, -1), target_grad=True,
                      k=k)
    assert den.grad.shape == den.shape and x.grad.shape == x.shape
    assert rel_l2(den.grad.cpu().numpy().ravel(), g.ravel()) <= 1e-14
    assert rel_l2(x.grad.cpu().numpy(), gt.sum(0)) <= 1e-13
