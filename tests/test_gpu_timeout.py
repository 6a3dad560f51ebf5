"""Failure detection on the device without a fault: a bounded wait that
runs out is reported as a status code, and the context stays usable.

The 3-D FP32-split kernels wait for each plane's TMA copy with a bounded
mbarrier wait.  The test arms the pipelined Runge-Kutta stage to first wait,
with a short bound, on a barrier phase that nothing completes (a flag that
nothing sets): the wait runs out, the kernel sets the timeout flag, waits
(with the default bound) for the copies it has in flight, and returns.  The
host then reports MISO_B200_ERR_TIMEOUT, where the reference would abort the
process (cuda_util.cuh:17-33), and a fresh handle on the same device steps
exactly as before.
"""
import numpy as np
import pytest

from miso_b200 import _lib
from miso_b200 import problems as P
from miso_b200.integrator import Integrator

pytestmark = pytest.mark.gpu


def _step(prob, nsteps, wait_limit=None):
    integ = Integrator(prob.config, prob.grid, sign=prob.sign, precision="fp32_split")
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    if wait_limit is not None:
        integ.set_wait_limit(wait_limit)
    try:
        for _ in range(nsteps):
            integ.update(integ.cfl())
        integ.sync()
        return integ.download()
    finally:
        integ.close()


def test_wait_that_runs_out_is_reported():
    prob = P.turbulence(32, seed=6)
    before = _step(prob, 2)
    integ = Integrator(prob.config, prob.grid, precision="fp32_split")
    integ.upload(prob.q)
    integ.apply_boundary_condition()
    assert integ.get_variant(0) == 3
    integ.arm_timeout_test(2_000_000)  # about 1 ms at the SM clock
    dt = integ.cfl()
    with pytest.raises(_lib.MisoError) as exc:
        integ.update(dt)
        integ.sync()
    assert exc.value.code == _lib.ERR_TIMEOUT
    integ.close()
    # the context is intact: a new handle steps bit for bit as before
    after = _step(prob, 2)
    assert np.array_equal(before, after)


def test_timeout_test_needs_the_pipelined_stage():
    prob = P.turbulence(24, seed=2)
    with Integrator(prob.config, prob.grid, precision="fp32_split") as integ:
        integ.set_variant(0, 1)
        with pytest.raises(_lib.MisoError) as exc:
            integ.arm_timeout_test(1000)
        assert exc.value.code == _lib.ERR_STATE


def test_wait_limit_default_restored():
    """A bound set back to the default (0) gives the normal step."""
    prob = P.turbulence(24, seed=2)
    ref = _step(prob, 1)
    assert np.array_equal(_step(prob, 1, wait_limit=0), ref)
