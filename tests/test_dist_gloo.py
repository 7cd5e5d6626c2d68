"""Right-hand-side replicas across ranks (fmmg_dist), as world-size-2 gloo
process groups on CPU.  The oracle stands in for each rank's GPU evaluate; the
gathered values must equal a single-process evaluation of every right-hand
side, and the step time must be the slowest rank's."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for _p in (os.path.join(ROOT, "fmm-g_b200"), os.path.join(ROOT, "oracle"), HERE):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import fmmg_dist  # noqa: E402


def test_rhs_blocks_cover_every_rhs_once():
    for k in (0, 1, 3, 8, 11):
        for world in (1, 2, 3, 8):
            got = []
            for r in range(world):
                first, count = fmmg_dist.rhs_block(k, world, r)
                got.extend(range(first, first + count))
            assert got == list(range(k))
    with pytest.raises(ValueError):
        fmmg_dist.rhs_block(4, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(k):
    rng = np.random.default_rng(20261203 + 77)
    src = rng.random((1500, 3))
    return src, rng.normal(size=(k, 1500))


def _worker(rank, world, port, k, out_dir):
    for _p in (os.path.join(ROOT, "fmm-g_b200"), os.path.join(ROOT, "oracle")):
        if _p not in sys.path:
            sys.path.insert(0, _p)
    import torch.distributed as dist
    import oracle as O
    import fmmg_dist as FD
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        src, dens = _problem(k)
        orc = O.Oracle(111, np_=4, pts_max=40)
        orc.setup(src, src, src)

        def block(d):
            rows = [torch.from_numpy(orc.evaluate(r.numpy()).ravel()) for r in d]
            return torch.stack(rows) if rows else torch.zeros((0, src.shape[0]), dtype=torch.float64)

        vals = FD.evaluate_replicated(block, torch.from_numpy(dens))
        slowest = FD.max_over_ranks(10.0 + rank)
        np.save(os.path.join(out_dir, "vals%d.npy" % rank), vals.numpy())
        np.save(os.path.join(out_dir, "t%d.npy" % rank), np.array([slowest]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("k", [3, 1])
def test_replicas_gather_every_rhs_and_take_the_slowest_rank(k, tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), k, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    import oracle as O
    src, dens = _problem(k)
    orc = O.Oracle(111, np_=4, pts_max=40)
    orc.setup(src, src, src)
    ref = np.stack([orc.evaluate(d).ravel() for d in dens])
    for r in range(world):
        vals = np.load(tmp_path / ("vals%d.npy" % r))
        assert vals.shape == ref.shape
        assert np.array_equal(vals, ref)  # the same oracle arithmetic, moved between ranks
        assert np.load(tmp_path / ("t%d.npy" % r))[0] == 10.0 + world - 1
