"""The bounded device waits and their error path.

Every mbarrier wait of the tensor-core kernels gives up after a time limit,
records an error flag and frees its tensor memory instead of spinning for
ever.  The self-test kernel waits on an mbarrier that nothing arrives on (no
tensor-core work is ever issued), with a short limit passed as a kernel
argument: the call must come back with FMMG_TIMEOUT, and the device must stay
usable for the evaluations that follow.
"""
import numpy as np
import pytest

import fmmg

pytestmark = pytest.mark.gpu


def test_wait_that_completes_returns_ok():
    assert fmmg.lib().fmmg_selftest_wait(0, 1, 1_000_000) == fmmg.FMMG_OK


@pytest.mark.parametrize("limit_ns", [0, 1000, 2_000_000])
def test_wait_that_runs_out_returns_timeout_and_the_device_stays_usable(limit_ns):
    assert fmmg.lib().fmmg_selftest_wait(0, 0, limit_ns) == fmmg.FMMG_TIMEOUT
    rng = np.random.default_rng(11)
    src = rng.random((3000, 3))
    den = rng.uniform(-1, 1, 3000)
    f = fmmg.FMM3d(111, np_=4, pts_max=40, device=0)
    f.setup(src)
    val = f.evaluate(den)
    rel, _, _ = f.check(den, val, np.arange(0, 3000, 7))
    assert rel < 1e-3
    assert f.device_error() == 0


def test_selftest_rejects_bad_limits():
    assert fmmg.lib().fmmg_selftest_wait(0, 0, -1) == fmmg.FMMG_INVALID_ARG
    assert fmmg.lib().fmmg_selftest_wait(0, 0, 3_000_000_000) == fmmg.FMMG_INVALID_ARG
