"""Finite-fault (focal) points in the CPU oracle: a focal point sampled every
half step whose series is m6 times a wavelet is the moment source with that
m6 and wavelet (every stage time falls on a sample, where the reference's
ExtractValue returns the sample itself), and a series that ends before the
run stops contributing."""
import dataclasses

import numpy as np

import models
import pyoracle
from helpers import comp_errors


def _run(m, steps):
    o = pyoracle.OracleSolver(m.desc(), 0)
    m.load(o)
    o.step(steps)
    seis = o.seismograms()[:, :, :steps]
    fw = np.stack([o.get_field(c) for c in range(9)])
    o.close()
    return seis, fw


def _as_focal(m):
    """The model's moment sources as focal points with fdt = stept/2."""
    n = len(m.mnt_loc)
    mom = np.einsum("qc,qt->cqt", m.mnt_m6.astype(np.float64), m.mnt_stf.astype(np.float64))
    return dataclasses.replace(m, mnt_loc=np.zeros((0, 3), np.int32),
                               mnt_m6=np.zeros((0, 6), np.float32),
                               mnt_stf=np.zeros((0, m.mnt_stf.shape[1]), np.float32),
                               foc_loc=m.mnt_loc.copy(), foc_mom=mom.astype(np.float32),
                               foc_dt=m.stept / 2), n


def test_focal_point_on_half_step_samples_is_the_moment_source():
    m = models.small_hill(nt=24, ni=18, nj=16, nk=14, nabs=(3, 4, 3, 3, 4, 0))
    mf, n = _as_focal(m)
    assert n >= 1
    s0, f0 = _run(m, 20)
    s1, f1 = _run(mf, 20)
    assert np.abs(s0).max() > 0
    # the focal series holds m6 x wavelet rounded to float32 (the moment source
    # multiplies them in FP64): agreement to float32 rounding, where a wrong
    # sample or time would be off by orders of magnitude
    for e in comp_errors(s1, s0):
        assert e < 1e-6
    for e in comp_errors(f1, f0):
        assert e < 1e-6


def test_focal_series_ends_contribute_nothing_after_their_window():
    m = models.small_hill(nt=30, ni=18, nj=16, nk=14, nabs=(3, 4, 3, 3, 4, 0))
    mf, _ = _as_focal(m)
    # keep the first 12 samples only (6 steps); the rest of the run is then
    # source-free, exactly as with a wavelet that is zero from sample 12 on
    cut = dataclasses.replace(mf, foc_mom=np.ascontiguousarray(mf.foc_mom[:, :, :12]))
    stf0 = m.mnt_stf.copy()
    stf0[:, 12:] = 0.0
    ref = dataclasses.replace(m, mnt_stf=stf0)
    s0, _ = _run(ref, 25)
    s1, _ = _run(cut, 25)
    for e in comp_errors(s1, s0):
        assert e < 1e-6
