"""The droplets driver (fmm3d_mpi/droplets.cpp) on the GPU: the right-hand
side through the evaluator in both forms against a dense Stokeslet sum at
sampled particles (a B200 gives 1.0e-6 FP64, 9.5e-7 mixed), and RK4 steps with
one handle set up again per right-hand side."""
import math

import numpy as np
import pytest

import droplets as D
import fmmg

pytestmark = pytest.mark.gpu


def _stokeslet_at(x, f, idx):
    """u_i = sum_{j != i} (I / r + r r^T / r^3) f_j / (8 pi) for i in idx."""
    out = []
    for c in range(0, len(idx), 100):
        d = x[idx[c:c + 100], None, :] - x[None, :, :]
        r2 = (d * d).sum(-1)
        self_ = r2 == 0.0
        r2[self_] = 1.0
        ir = 1.0 / np.sqrt(r2)
        ir[self_] = 0.0
        rf = (d * f[None, :, :]).sum(-1)
        out.append(ir.dot(f) + (d * (rf * ir ** 3)[:, :, None]).sum(1))
    return np.concatenate(out) / (8.0 * math.pi)


def _rhs_error(precision, x, eps, idx):
    d = D.Droplets(x, eps, 0.1, velocity=D.FmmVelocity(np_=6, pts_max=64, precision=precision))
    k = d.rhs(d.x).cpu().numpy()
    f = np.zeros_like(x)
    f[:, 2] = -eps * eps
    want = f[idx] + 6.0 * math.pi * eps * _stokeslet_at(x, f, idx)
    return np.linalg.norm(k[idx] - want) / np.linalg.norm(want), k


def test_droplets_rhs_both_forms_against_dense_sum():
    x = D.snap_and_dedup(D.initial_positions(60000, "two_balls_vert"))
    eps = D.particle_size(x.shape[0], 0.1)
    idx = np.random.default_rng(11).choice(x.shape[0], 500, replace=False)
    e64, k64 = _rhs_error(fmmg.PREC_FP64, x, eps, idx)
    emx, kmx = _rhs_error(fmmg.PREC_MIXED, x, eps, idx)
    print("droplets rhs vs dense: fp64 %.3e mixed %.3e" % (e64, emx))
    assert e64 <= 1e-5 and emx <= 1e-4


def test_droplets_rk4_steps_on_one_handle():
    x = D.initial_positions(20000, "ball")
    eps = D.particle_size(x.shape[0], 0.05)
    vel = D.FmmVelocity(np_=4, pts_max=64)
    d = D.Droplets(x, eps, 0.5, velocity=vel)
    z0 = d.x[:, 2].mean().item()
    d.run(2)
    assert d.evaluations == 8
    xn = d.x.cpu().numpy()
    assert np.isfinite(xn).all()
    assert xn[:, 2].mean() < z0
