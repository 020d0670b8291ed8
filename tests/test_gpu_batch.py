"""Batched models and the work-list autotuner.

A batch steps several independent models through one persistent launch per
stage part; its per-cell arithmetic is the single-model kernel's source, so
every member's seismograms and fields must equal those of the same model run
alone up to FP32 rounding (the batched instantiation is a separate
compilation; measured <= 9.3e-7 relative L2 per component over 24 steps, held
to the 1e-5 parity bar).  The autotuner changes the work list (tile order
and z-chunking) of the same kernels and the launch shape (one persistent
launch, or every member's own single-model step graphs), so it must leave
the state unchanged and the results within that bar.
"""
import numpy as np
import pytest

import cgfd
import models
from helpers import comp_errors

pytestmark = pytest.mark.gpu


def _small_batch(n=3, nt=30):
    return models.batch_models(n=n, seed=11, nt=nt, side=(28, 44), nabs_cells=5)


def _alone(m, steps):
    s = cgfd.Solver(m.desc())
    m.load(s)
    s.step(steps)
    out = (s.seismograms(), np.stack([s.get_field(c) for c in range(9)]))
    s.close()
    return out


def test_batch_members_equal_single_model_runs():
    ms = _small_batch()
    steps = 24
    ref = [_alone(m, steps) for m in ms]
    b = cgfd.Batch([m.desc() for m in ms])
    for m, s in zip(ms, b.models):
        m.load(s)
    b.step(steps)
    b.sync()
    for q, s in enumerate(b.models):
        seis = s.seismograms()
        fw = np.stack([s.get_field(c) for c in range(9)])
        for c, e in enumerate(comp_errors(seis, ref[q][0])):
            assert e < 1e-5, (q, cgfd.COMPONENTS[c], e)
        for c, e in enumerate(comp_errors(fw, ref[q][1])):
            assert e < 1e-5, (q, cgfd.COMPONENTS[c], e)
    b.close()


def test_batch_steps_in_chunks_like_one_call():
    ms = _small_batch(n=2)
    b1 = cgfd.Batch([m.desc() for m in ms])
    b2 = cgfd.Batch([m.desc() for m in ms])
    for bb in (b1, b2):
        for m, s in zip(ms, bb.models):
            m.load(s)
    b1.step(20)
    for _ in range(4):
        b2.step(5)
    for s1, s2 in zip(b1.models, b2.models):
        assert np.array_equal(s1.seismograms(), s2.seismograms())
    b1.close()
    b2.close()


def test_autotune_keeps_state_and_results():
    m = models.small_hill(nt=40)
    s = cgfd.Solver(m.desc())
    m.load(s)
    s.step(10)
    before = np.stack([s.get_field(c) for c in range(9)])
    ms = s.autotune(steps=2)
    assert ms > 0
    after = np.stack([s.get_field(c) for c in range(9)])
    assert np.array_equal(before, after)
    s.step(10)
    ref = cgfd.Solver(m.desc())
    m.load(ref)
    ref.step(20)
    assert np.array_equal(s.seismograms(), ref.seismograms())
    s.close()
    ref.close()


def test_work_shape_is_readable_settable_and_leaves_results_bit_equal():
    """The work-list shape (cgfd_get/set_work_shape) changes only which CTA
    computes which (tile, z-chunk) item: the results stay bit-equal."""
    m = models.small_hill(nt=40)
    a = cgfd.Solver(m.desc())
    m.load(a)
    a.prepare()
    assert a.work_shape == (6, 16, 1.0)  # the default
    a.work_shape = (3, 12, 2.0)
    assert a.work_shape == (3, 12, 2.0)
    with pytest.raises(cgfd.CgfdError):
        a.work_shape = (0, 12, 1.0)
    a.step(20)
    b = cgfd.Solver(m.desc())
    m.load(b)
    b.step(20)
    assert np.array_equal(a.seismograms(), b.seismograms())
    a.close()
    b.close()


def test_batch_autotune_keeps_results():
    ms = _small_batch(n=2, nt=30)
    b = cgfd.Batch([m.desc() for m in ms])
    for m, s in zip(ms, b.models):
        m.load(s)
    b.step(5)
    assert b.autotune(steps=1) > 0
    b.step(10)
    for m, s in zip(ms, b.models):
        seis, _ = _alone(m, 15)
        for c, e in enumerate(comp_errors(s.seismograms()[:, :, :15], seis[:, :, :15])):
            assert e < 1e-5, (cgfd.COMPONENTS[c], e)
    b.close()


@pytest.mark.parametrize("storage", [cgfd.STORE_F32, cgfd.STORE_F16])
def test_member_launch_equals_single_model_runs_bit_for_bit(storage):
    """The member launch shape runs every member's own step graphs (the
    single-model kernels), so members equal the same models run alone bit
    for bit, 16-bit storage included, over steps taken in several calls."""
    ms = _small_batch(n=2)
    steps = 12

    def alone(m):
        s = cgfd.Solver(m.desc(storage=storage))
        m.load(s)
        s.step(steps)
        out = (s.seismograms(), np.stack([s.get_field(c) for c in range(9)]))
        s.close()
        return out

    ref = [alone(m) for m in ms]
    b = cgfd.Batch([m.desc(storage=storage) for m in ms])
    for m, s in zip(ms, b.models):
        m.load(s)
    assert b.launch == cgfd.BATCH_PERSISTENT
    b.launch = cgfd.BATCH_MEMBERS
    assert b.launch == cgfd.BATCH_MEMBERS
    b.step(steps // 2)
    b.step(steps - steps // 2)
    b.sync()
    for q, s in enumerate(b.models):
        assert np.array_equal(s.seismograms(), ref[q][0]), q
        assert np.array_equal(np.stack([s.get_field(c) for c in range(9)]), ref[q][1]), q
    with pytest.raises(cgfd.CgfdError):
        b.launch = 7
    b.close()
