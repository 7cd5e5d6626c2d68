"""The droplets driver (fmm3d_mpi/droplets.cpp) on CPU: its generator and
initial particles against the reference's own loop run with the C library's
drand48, the snapping and de-duplication, the right-hand side against a dense
Stokeslet sum (the oracle standing in for the GPU evaluate), and the RK4 step.
"""
import ctypes
import math

import numpy as np
import pytest
import torch

import droplets as D
import oracle as O


def _libc():
    libc = ctypes.CDLL(None)
    libc.drand48.restype = ctypes.c_double
    libc.srand48.argtypes = [ctypes.c_long]
    return libc


@pytest.mark.parametrize("seed", [0, 1, 7, 2 ** 31 + 5])
def test_drand48_restatement_equals_the_c_library(seed):
    libc = _libc()
    libc.srand48(seed)
    ref = np.array([libc.drand48() for _ in range(9000)])
    np.testing.assert_array_equal(D.Drand48(seed).draws(9000), ref)


def _reference_loop(n, distribution, seed=0):
    """droplets.cpp:203, 251-300 as written, with the C library's drand48."""
    libc = _libc()
    libc.srand48(seed)
    out = np.zeros((n, 3))

    def fill(k0, k1, dz):
        k = k0
        while k < k1:
            tmp = [1 - 2 * libc.drand48() for _ in range(3)]
            if sum(t * t for t in tmp) >= 1:
                continue
            out[k] = tmp
            out[k, 2] += dz
            k += 1

    if distribution == "ball":
        fill(0, n, 0.0)
    else:
        fill(0, n // 2, 0.0)
        fill(n // 2, n, 4.0)
    return out


@pytest.mark.parametrize("distribution", ["ball", "two_balls_vert"])
def test_initial_particles_are_the_reference_loops(distribution):
    for n in (1, 301, 2000):
        np.testing.assert_array_equal(D.initial_positions(n, distribution), _reference_loop(n, distribution))
    with pytest.raises(ValueError):
        D.initial_positions(10, "cube")


def test_snap_and_dedup():
    x = D.initial_positions(3000, "two_balls_vert")
    x = np.concatenate([x, x[:50], x[100:101]])  # exact duplicates
    y = D.snap_and_dedup(x)
    assert y.shape == (3000, 3)
    scale, shift = D.box_map(x)
    u = np.ldexp((y + shift) * scale, 30)
    # cell centres of the scaled frame, distinct, moved by at most half a cell
    np.testing.assert_allclose(u - np.floor(u), 0.5, atol=1e-5)
    cells = np.floor(u).astype(np.uint64)
    keys = D._morton(cells)
    assert np.all(keys[1:] > keys[:-1]), "Morton order, no duplicates"
    # each snapped point is its original one, sorted by the key of its cell
    orig = x[:3000]
    order = np.argsort(D._morton(np.ldexp((orig + shift) * scale, 30).astype(np.uint64)))
    assert np.abs(y - orig[order]).max() <= 2.0 ** -30 / scale
    # z is the most significant axis of a level, then y, then x
    c = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1]], dtype=np.uint64)
    assert D._morton(c).tolist() == [1, 2, 4, 7]


def _stokeslet_dense(x, f):
    """u_i = sum_{j != i} (I / r + r r^T / r^3) f_j / (8 pi), mu = 1."""
    d = x[:, None, :] - x[None, :, :]
    r2 = (d * d).sum(-1)
    np.fill_diagonal(r2, 1.0)
    ir = 1.0 / np.sqrt(r2)
    np.fill_diagonal(ir, 0.0)
    rf = (d * f[None, :, :]).sum(-1)
    u = ir.dot(f) + (d * (rf * ir ** 3)[:, :, None]).sum(1)
    return u / (8.0 * math.pi)


class _OracleVelocity:
    device = torch.device("cpu")

    def __init__(self, np_=6, pts_max=64):
        self.np_, self.pts_max = np_, pts_max

    def __call__(self, xs, den):
        x = xs.numpy()
        o = O.Oracle(D.KERNEL, np_=self.np_, pts_max=self.pts_max)
        o.setup(x, x, x)
        return torch.from_numpy(o.evaluate(den.numpy()).reshape(-1, 3))


class _DenseVelocity:
    device = torch.device("cpu")

    def __call__(self, xs, den):
        return torch.from_numpy(_stokeslet_dense(xs.numpy(), den.numpy().reshape(-1, 3)))


def test_rhs_is_force_plus_scaled_fmm_velocity():
    x = D.snap_and_dedup(D.initial_positions(2500, "ball"))
    eps = D.particle_size(x.shape[0], 0.1)
    d = D.Droplets(x, eps, 0.1, velocity=_OracleVelocity())
    k = d.rhs(d.x).numpy()
    f = np.zeros_like(x)
    f[:, 2] = -eps * eps
    want = f + 6.0 * math.pi * eps * _stokeslet_dense(x, f)  # in the caller's coordinates
    rel = np.linalg.norm(k - want) / np.linalg.norm(want)
    assert rel < 1e-5, rel
    # a cloud settles faster than one particle alone (whose k is its force)
    assert k[:, 2].mean() < -1.5 * eps * eps
    assert d.evaluations == 1


def test_rk4_step_on_a_linear_field():
    rng = np.random.default_rng(0)
    A = torch.from_numpy(rng.normal(size=(3, 3)))
    x0 = torch.from_numpy(rng.normal(size=(50, 3)))
    h = 0.05
    got = D.rk4_step(x0, lambda x: x @ A.T, h)
    hA = h * A
    P = torch.eye(3, dtype=torch.float64) + hA + hA @ hA / 2 + hA @ hA @ hA / 6 + hA @ hA @ hA @ hA / 24
    torch.testing.assert_close(got, x0 @ P.T, rtol=0, atol=1e-14)


def test_run_writes_positions(tmp_path):
    x = D.initial_positions(200, "two_balls_vert")
    d = D.Droplets(x, 0.05, 0.2, velocity=_DenseVelocity())
    z0 = d.x[:, 2].mean().item()
    d.run(3, write_fraction=2, out_dir=str(tmp_path))
    assert sorted(p.name for p in tmp_path.iterdir()) == ["coord0.txt", "coord2.txt"]
    np.testing.assert_array_equal(np.loadtxt(tmp_path / "coord0.txt"), x)
    assert np.loadtxt(tmp_path / "coord2.txt").shape == (200, 3)
    assert d.evaluations == 12
    assert d.x[:, 2].mean().item() < z0  # the particles sink


def test_command_line(tmp_path, monkeypatch, capsys):
    """main() with the reference's options, a dense CPU stand-in for the GPU
    evaluator: eps from -volume_ratio, positions written every
    -write_fraction steps, the timing line printed."""
    class Stand(_DenseVelocity):
        def __init__(self, np_, pts_max, precision):
            self.setup_s = self.evaluate_s = 0.0

    monkeypatch.setattr(D, "FmmVelocity", Stand)
    D.main(["--numsrc", "150", "--distribution", "ball", "--time_step", "0.1", "--volume_ratio", "0.2",
            "--num_iter", "2", "--write_fraction", "1", "--out", str(tmp_path), "--preserve_order"])
    out = capsys.readouterr().out
    n = D.snap_and_dedup(D.initial_positions(150, "ball")).shape[0]
    assert "particles %d, particle size %g" % (n, D.particle_size(n, 0.2)) in out
    assert "2 steps (8 right-hand sides)" in out
    assert sorted(p.name for p in tmp_path.iterdir()) == ["coord0.txt", "coord1.txt", "coord2.txt"]
    with pytest.raises(SystemExit):  # -particle_size and -volume_ratio exclude each other
        D.main(["--numsrc", "10", "--distribution", "ball", "--time_step", "0.1", "--volume_ratio", "0.2",
                "--particle_size", "0.01", "--num_iter", "1", "--write_fraction", "1"])
