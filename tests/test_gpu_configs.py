"""The other benchmark configurations as test cases, at reduced sizes with
their geometry, kernels, np and k: each form against the FP64 dense sum
(sampled targets, as the reference check() does), and the mixed form against
the FP64 form.  Observed errors are printed; the bounds sit a few times above
what a B200 gives (config3: FP64 3.6e-5, mixed 4.6e-5, mixed vs FP64 6.0e-6;
config5: FP64 9.3e-8, mixed 4.8e-6; config1 at np 4: 1.24e-4 in both forms,
the truncation error of order 4)."""
import numpy as np
import pytest

import fmmg
import workloads as W
from gpu_common import rel_l2

pytestmark = pytest.mark.gpu


def _run(cfg, k, precision, n_chk=2000, coefs=(1.0, 0.25)):
    import torch
    n = cfg["src"].shape[0]
    f = fmmg.FMM3d(cfg["kernel"], np_=cfg["np"], pts_max=cfg["pts_max"], coefs=coefs)
    f.setup(cfg["src"], cfg["nrm"])
    den = np.atleast_2d(cfg["den"])[:k]
    d = torch.from_numpy(np.ascontiguousarray(den)).cuda()
    out = torch.zeros(k, n * f.td, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    f.evaluate_device(d, out, k, precision)
    f.sync()
    vals = out.cpu().numpy()
    idx = np.random.default_rng(7).choice(n, n_chk, replace=False)
    errs = [f.check(den[r], vals[r], idx)[0] for r in (0, k - 1)]
    return f, vals, errs


def test_config3_stokes_double_layer_ellipsoids_mixed_k8():
    cfg = W.config3(n=150000, k_rhs=8)
    _, vm, em = _run(cfg, 8, fmmg.PREC_MIXED)
    _, vd, ed = _run(cfg, 8, fmmg.PREC_FP64)
    print("config3 mixed %s fp64 %s mixed-vs-fp64 %.3e" % (em, ed, rel_l2(vm, vd)))
    assert max(ed) <= 1e-4 and max(em) <= 1e-4
    assert rel_l2(vm, vd) <= 3e-5


def test_config5_navier_np8_mixed():
    cfg = W.config5(n=120000, k_rhs=4)
    _, vm, em = _run(cfg, 4, fmmg.PREC_MIXED, coefs=(1.0, 0.3))
    _, vd, ed = _run(cfg, 4, fmmg.PREC_FP64, coefs=(1.0, 0.3))
    print("config5 mixed %s fp64 %s mixed-vs-fp64 %.3e" % (em, ed, rel_l2(vm, vd)))
    assert max(ed) <= 1e-6
    assert max(em) <= 2e-5


def test_config1_laplace_uniform_np4_both_forms():
    cfg = W.config1()
    _, vm, em = _run(cfg, 1, fmmg.PREC_MIXED)
    _, vd, ed = _run(cfg, 1, fmmg.PREC_FP64)
    print("config1 mixed %s fp64 %s mixed-vs-fp64 %.3e" % (em, ed, rel_l2(vm, vd)))
    assert max(ed) <= 3e-4 and max(em) <= 3e-4
    assert rel_l2(vm, vd) <= 1e-5
