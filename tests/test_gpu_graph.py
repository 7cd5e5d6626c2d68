"""CUDA-graph replay of evaluate_device: the captured evaluate must give the
same values as the eager one, read the densities written into the captured
buffers at replay time, and start over when the buffers change."""
import numpy as np
import pytest

import fmmg
import workloads as W
from gpu_common import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,k", [(fmmg.PREC_FP64, 1), (fmmg.PREC_MIXED, 1), (fmmg.PREC_MIXED, 8)])
def test_graph_replay_matches_eager(precision, k):
    import torch
    rng = np.random.default_rng(31 + k)
    n = 40000
    src = W.sphere_clusters(n, rng)
    f = fmmg.FMM3d(111, np_=6, pts_max=64)
    f.setup(src)
    d1 = rng.normal(size=(k, n))
    d2 = rng.normal(size=(k, n))

    def eager(d):
        out = torch.zeros(k, n, dtype=torch.float64, device="cuda")
        f.set_graph(False)
        f.evaluate_device(torch.from_numpy(d).cuda(), out, k, precision)
        f.sync()
        return out.cpu().numpy()

    ref1, ref2 = eager(d1), eager(d2)
    f.set_graph(True)
    den = torch.from_numpy(d1).cuda()
    out = torch.zeros(k, n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for call in range(3):  # eager, capture + launch, replay
        out.zero_()
        torch.cuda.synchronize()
        f.evaluate_device(den, out, k, precision)
        f.sync()
        assert rel_l2(out.cpu().numpy(), ref1) == 0.0, call
    active, note = f.graph_state()
    assert active, note
    den.copy_(torch.from_numpy(d2))  # new densities in the captured buffer
    torch.cuda.synchronize()
    f.evaluate_device(den, out, k, precision)
    f.sync()
    assert rel_l2(out.cpu().numpy(), ref2) == 0.0
    out2 = torch.zeros(k, n, dtype=torch.float64, device="cuda")  # another output buffer: a new key
    torch.cuda.synchronize()
    for _ in range(3):
        f.evaluate_device(den, out2, k, precision)
        f.sync()
    assert rel_l2(out2.cpu().numpy(), ref2) == 0.0
    assert f.graph_state()[0]
