"""The autotuner picks launch shapes by timing real evaluates; the shapes
change how work is split across CTAs, never which terms are summed."""
import numpy as np
import pytest

import fmmg
import workloads as W
from gpu_common import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,k", [(fmmg.PREC_FP64, 1), (fmmg.PREC_MIXED, 8)])
def test_autotune_picks_candidates_and_keeps_results(precision, k):
    import torch
    rng = np.random.default_rng(61 + k)
    n = 60000
    f = fmmg.FMM3d(111, np_=6, pts_max=64)
    f.setup(W.sphere_clusters(n, rng))
    den = torch.from_numpy(rng.normal(size=(k, n))).cuda()
    out = torch.zeros(k, n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    f.evaluate_device(den, out, k, precision)
    f.sync()
    before = out.cpu().numpy()
    ms, tune = f.autotune(den, out, k, precision, reps=1)
    assert ms > 0
    assert tune["had_rows_fp32"] in (32, 64, 128, 256) and tune["had_rows_fp64"] in (32, 64, 128, 256)
    assert tune["gemm_split_ctas_per_sm"] in (0, 1, 2, 4)
    out.zero_()
    torch.cuda.synchronize()
    f.evaluate_device(den, out, k, precision)
    f.sync()
    after = out.cpu().numpy()
    if precision == fmmg.PREC_FP64:
        assert np.array_equal(after, before)  # FP64 sums never depend on the shapes
    else:
        assert rel_l2(after, before) <= 1e-6  # split-K may reorder FP32 sums
    f.tuning({"had_rows_fp32": 64, "had_rows_fp64": 128, "gemm_split_ctas_per_sm": 2})
    assert f.tuning()["had_rows_fp64"] == 128
