"""Seeded synthetic inputs with the shapes of the benchmark configurations.

The reference measures on no public dataset; these generators stand in for the
point distributions of its driver (fmm3d_mpi/tt0.cpp:209-298): uniform in the
unit box, points on a sphere of radius 0.49 about the centre, Gaussian clusters
resampled until they fall inside [0, 1)^3 (tt0.cpp:235-241), and unit normals.
Seeds are 20261203 + config number.
"""
import numpy as np

SEED = 20261203


def unit_normals(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1)[:, None]


def _inside(p):
    return ((p >= 0.0) & (p < 1.0)).all(axis=1)


def uniform(n, rng):
    return rng.random((n, 3))


def sphere(n, rng, radius=0.49, ctr=0.5):
    v = rng.normal(size=(n, 3))
    return ctr + radius * v / np.linalg.norm(v, axis=1)[:, None]


def clusters(n, rng, k=8, sigma=0.02, lo=0.1, hi=0.9):
    centres = rng.uniform(lo, hi, size=(k, 3))
    out = centres[rng.integers(0, k, n)] + sigma * rng.normal(size=(n, 3))
    bad = ~_inside(out)
    while bad.any():
        m = int(bad.sum())
        out[bad] = centres[rng.integers(0, k, m)] + sigma * rng.normal(size=(m, 3))
        bad = ~_inside(out)
    return out


def sphere_clusters(n, rng):
    """Config 2 geometry: 50% on the sphere surface, 50% in 8 Gaussian clusters."""
    m = n // 2
    return np.concatenate([sphere(m, rng), clusters(n - m, rng)])


def config1(n=65536):
    """Laplace S, uniform points, densities U[-1, 1], np=4, ptsMax=150."""
    rng = np.random.default_rng(SEED + 1)
    src = uniform(n, rng)
    return dict(kernel=111, np=4, pts_max=150, src=src, nrm=src, den=rng.uniform(-1, 1, n))


def config2(n=1 << 20):
    """Laplace S, sphere + clusters, densities N(0, 1), np=6, ptsMax=64."""
    rng = np.random.default_rng(SEED + 2)
    src = sphere_clusters(n, rng)
    return dict(kernel=111, np=6, pts_max=64, src=src, nrm=src, den=rng.normal(size=n))


def ellipsoids(n, rng, k=64):
    """Points uniform in area on k random ellipsoids with outward unit normals."""
    axes = rng.uniform(0.02, 0.08, size=(k, 3))
    ctr = rng.uniform(0.1, 0.9, size=(k, 3))
    q = rng.normal(size=(k, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    w, x, y, z = q.T
    R = np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
                  np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
                  np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], 1)
    pts, nrm = [], []
    per = np.full(k, n // k)
    per[: n - per.sum()] += 1
    for e in range(k):
        a = axes[e]
        got_p, got_n = [], []
        need = per[e]
        while need > 0:
            u = rng.normal(size=(2 * need + 16, 3))
            u /= np.linalg.norm(u, axis=1)[:, None]
            # area element of the map u -> a*u relative to its maximum (rejection)
            g = np.sqrt((u[:, 0] * a[1] * a[2]) ** 2 + (u[:, 1] * a[0] * a[2]) ** 2 + (u[:, 2] * a[0] * a[1]) ** 2)
            keep = rng.random(len(u)) < g / g.max()
            u = u[keep][:need]
            p = u * a
            nn = p / a ** 2
            nn /= np.linalg.norm(nn, axis=1)[:, None]
            got_p.append(p @ R[e].T + ctr[e])
            got_n.append(nn @ R[e].T)
            need -= len(u)
        pts.append(np.concatenate(got_p))
        nrm.append(np.concatenate(got_n))
    return np.clip(np.concatenate(pts), 0.0, 1.0), np.concatenate(nrm)


def config3(n=1 << 20, k_rhs=8):
    """Stokes D_U (mu = 1) on 64 ellipsoids, 3-vector densities N(0, 1), np=6."""
    rng = np.random.default_rng(SEED + 3)
    src, nrm = ellipsoids(n, rng)
    return dict(kernel=321, np=6, pts_max=64, src=src, nrm=nrm, den=rng.normal(size=(k_rhs, 3 * n)))


def config4(n=1 << 22, k_rhs=16):
    """Laplace S adjoint case: uniform points, k_rhs densities N(0, 1), np=6."""
    rng = np.random.default_rng(SEED + 4)
    src = uniform(n, rng)
    return dict(kernel=111, np=6, pts_max=64, src=src, nrm=src, den=rng.normal(size=(k_rhs, n)))


def config5(n=1 << 21, k_rhs=32):
    """Navier S_U (mu 1, nu 0.3): 70% uniform, 30% on a shell r = 0.3 +- 0.001, np=8."""
    rng = np.random.default_rng(SEED + 5)
    m = int(0.7 * n)
    a = uniform(m, rng)
    v = rng.normal(size=(n - m, 3))
    r = rng.uniform(0.299, 0.301, size=(n - m, 1))
    b = 0.5 + r * v / np.linalg.norm(v, axis=1)[:, None]
    src = np.concatenate([a, b])
    return dict(kernel=511, np=8, pts_max=64, coefs=(1.0, 0.3), src=src, nrm=src,
                den=rng.uniform(-1, 1, size=(k_rhs, 3 * n)))
