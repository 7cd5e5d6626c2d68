"""Right-hand-side replicas (fmmg_dist) with the GPU handle as each rank's
evaluator: two ranks of a gloo process group (host-side collectives) share
cuda:0, each with its own handle on its own stream, and evaluate their own
blocks of the right-hand sides.  The gathered values must equal one handle's
evaluation of every right-hand side (the FP64 form evaluates the right-hand
sides one at a time: the same arithmetic on either side), and the reported
step time must be the slowest rank's.  No kernel of one rank waits on the
other: only the host collectives meet."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if os.path.join(ROOT, "fmm-g_b200") not in sys.path:
    sys.path.insert(0, os.path.join(ROOT, "fmm-g_b200"))

pytestmark = pytest.mark.gpu

K = 5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem():
    rng = np.random.default_rng(20261204)
    src = rng.random((40000, 3))
    return src, rng.normal(size=(K, src.shape[0]))


def _worker(rank, world, port, out_dir):
    if os.path.join(ROOT, "fmm-g_b200") not in sys.path:
        sys.path.insert(0, os.path.join(ROOT, "fmm-g_b200"))
    import datetime
    import torch.distributed as dist
    import fmmg
    import fmmg_dist as FD
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        src, dens = _problem()
        f = fmmg.FMM3d(111, np_=5, pts_max=48, device=0)
        f.setup(src)
        n = src.shape[0]

        def block(d):
            out = torch.zeros((d.shape[0], n), dtype=torch.float64, device="cuda")
            if d.shape[0]:
                f.evaluate_device(d.to("cuda").contiguous(), out, k=d.shape[0], precision=fmmg.PREC_FP64)
                f.sync()
            return out.cpu()

        vals = FD.evaluate_replicated(block, torch.from_numpy(dens))
        slowest = FD.max_over_ranks(3.0 + 2.0 * rank)
        np.save(os.path.join(out_dir, "vals%d.npy" % rank), vals.numpy())
        np.save(os.path.join(out_dir, "t%d.npy" % rank), np.array([slowest]))
        f.close()
    finally:
        dist.destroy_process_group()


def test_gpu_handles_as_replicas_gather_every_rhs(tmp_path):
    import fmmg
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    src, dens = _problem()
    f = fmmg.FMM3d(111, np_=5, pts_max=48, device=0)
    f.setup(src)
    d = torch.from_numpy(dens).cuda()
    out = torch.zeros_like(d)
    f.evaluate_device(d, out, k=K, precision=fmmg.PREC_FP64)
    f.sync()
    want = out.cpu().numpy()
    for r in range(world):
        got = np.load(os.path.join(str(tmp_path), "vals%d.npy" % r))
        assert got.shape == want.shape
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
        assert float(np.load(os.path.join(str(tmp_path), "t%d.npy" % r))[0]) == 5.0
