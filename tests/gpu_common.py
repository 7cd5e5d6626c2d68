"""Shared helpers for the GPU tests: seeded synthetic inputs and the oracle runs."""
import numpy as np

import fmmg
import oracle as O

SEED = 20261203


def unit_normals(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1)[:, None]


def points(kind, n, rng):
    """Synthetic distributions with the shapes of the benchmark configs."""
    if kind == "uniform":
        return rng.random((n, 3))
    if kind == "sphere_clusters":  # half on a sphere (r 0.49 about the centre), half in 8 Gaussian clusters
        m = n // 2
        v = rng.normal(size=(m, 3))
        s = 0.5 + 0.49 * v / np.linalg.norm(v, axis=1)[:, None]
        ctr = rng.uniform(0.1, 0.9, size=(8, 3))
        c = ctr[rng.integers(0, 8, n - m)] + 0.02 * rng.normal(size=(n - m, 3))
        bad = (c < 0) | (c >= 1)
        while bad.any():
            rows = bad.any(axis=1)
            c[rows] = ctr[rng.integers(0, 8, rows.sum())] + 0.02 * rng.normal(size=(rows.sum(), 3))
            bad = (c < 0) | (c >= 1)
        return np.concatenate([s, c])
    raise ValueError(kind)


def share_operators(lib, orc):
    """Give the oracle the library's operator tables (the 1e-10 parity gate
    compares the two evaluate() implementations on identical operators)."""
    for which, idxs in ((0, [0]), (1, range(8)), (2, [0]), (3, range(8)), (4, range(316))):
        for i in idxs:
            orc.set_operator(which, i, lib.operator(which, i))


def rel_l2(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def gpu_eval(lib, den, stages=fmmg.STAGE_ALL):
    import torch
    d = torch.from_numpy(np.ascontiguousarray(den, dtype=np.float64).ravel()).cuda()
    out = torch.zeros(lib.nt * lib.td, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    if stages == fmmg.STAGE_ALL:
        lib.evaluate_device(d, out)
    else:
        lib.evaluate_stages(d, out, stages)
    torch.cuda.synchronize()
    lib.sync()
    return out.cpu().numpy()
