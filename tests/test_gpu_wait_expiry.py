"""The bounded device waits of the stage kernels (failure detection without a
GPU fault).  Every mbarrier wait of the default kernel gives up after a
limit; cgfd_test_withhold_copy shortens the limit to a few milliseconds and
makes the velocity part's first CTA withhold one tensor copy, so that its
wait for that plane runs out: nothing faults or hangs, the CTA records the
expiry, drains its own copies (bounded) and returns, and cgfd_sync reports
CGFD_ERR_TIMEOUT.  A new solver on the same device then runs normally (its
seismograms equal the FP64 oracle's)."""
import time

import numpy as np
import pytest

import cgfd
import models
import pyoracle
from helpers import comp_errors

pytestmark = pytest.mark.gpu


def test_expired_wait_reports_timeout_and_the_device_stays_usable():
    m = models.small_flat(nt=12)
    s = cgfd.Solver(m.desc(kernel=cgfd.KERNEL_FUSED))
    m.load(s)
    s.prepare()
    s.test_withhold_copy(0.005, 2)
    t0 = time.perf_counter()
    s.step(1)
    with pytest.raises(cgfd.CgfdError) as ei:
        s.sync(timeout_s=60.0)
    assert ei.value.status == cgfd.ERR_TIMEOUT
    assert "bounded wait" in str(ei.value)
    assert time.perf_counter() - t0 < 30.0
    s.close()

    m2 = models.small_flat(nt=10)
    p = cgfd.Solver(m2.desc(kernel=cgfd.KERNEL_FUSED))
    m2.load(p)
    p.step(10)
    p.sync()
    got = p.seismograms()
    p.close()
    o = pyoracle.OracleSolver(m2.desc(), 0)
    m2.load(o)
    o.step(10)
    ref = o.seismograms()
    o.close()
    assert np.abs(ref[:3]).max() > 0
    for c, e in enumerate(comp_errors(got, ref)):
        assert e < 1e-5, (cgfd.COMPONENTS[c], e)


def test_withhold_hook_checks_its_arguments_and_restores():
    m = models.small_flat(nt=6)
    s = cgfd.Solver(m.desc(kernel=cgfd.KERNEL_FUSED))
    m.load(s)
    for bad in (0.0, -1.0, 61.0):
        with pytest.raises(cgfd.CgfdError):
            s.test_withhold_copy(bad, 2)
    s.test_withhold_copy(0.005, 2)
    s.test_withhold_copy(1.0, -1)  # restored before any step ran
    s.step(6)
    s.sync()
    assert s.check_finite() == 0
    s.close()
    q = cgfd.Solver(m.desc(kernel=cgfd.KERNEL_SIMPLE))
    with pytest.raises(cgfd.CgfdError):
        q.test_withhold_copy(0.005, 2)
    q.close()
