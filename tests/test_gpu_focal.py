"""Finite-fault (focal) points on the GPU (cgfd_upload_focal): the series
are interpolated on the device every stage, as the reference's InterpFocus /
ExtractValue do on the host, and injected like its LoadRmom.  Against the
FP64 oracle within the 1e-5 parity bar (all kernel families, whole steps and
single stages), in a batch against the same models alone, and with 16-bit
storage against FP32 storage."""
import dataclasses

import numpy as np
import pytest

import cases
import cgfd
import models
import pyoracle
from helpers import comp_errors, valid

pytestmark = pytest.mark.gpu

TOL = 1e-5
KERNELS = [cgfd.KERNEL_SIMPLE, cgfd.KERNEL_FUSED, cgfd.KERNEL_SCALAR]
KIDS = ["simple", "fused", "scalar"]


def _fault_model(nt=40):
    m = models.small_hill(nt=nt, nabs=(5, 6, 4, 5, 5, 0))
    # the fault replaces the point sources; centre 8 cells below the surface
    m = dataclasses.replace(m, mnt_loc=np.zeros((0, 3), np.int32),
                            mnt_m6=np.zeros((0, 6), np.float32),
                            mnt_stf=np.zeros((0, m.mnt_stf.shape[1]), np.float32))
    return models.with_finite_fault(m, center=(3 + m.ni // 2, 3 + m.nj // 2, 3 + m.nk - 9),
                                    length=6, width=4, m0=1e15, vr=2500.0, rise=0.06)


def _fields(s, fset=0):
    return np.stack([s.get_field(c, fset) for c in range(9)])


@pytest.mark.parametrize("kernel", KERNELS, ids=KIDS)
def test_finite_fault_matches_fp64_oracle(kernel):
    m = _fault_model()
    assert m.foc_mom.shape[1] == 24 and abs(m.foc_dt - 1.7 * m.stept) < 1e-12
    steps = 36
    p = cgfd.Solver(m.desc(kernel=kernel))
    m.load(p)
    p.step(steps)
    o = pyoracle.OracleSolver(m.desc(), 0)
    m.load(o)
    o.step(steps)
    ps, os_ = p.seismograms()[:, :, :steps], o.seismograms()[:, :, :steps]
    assert np.abs(os_[:3]).max() > 0
    for c, e in enumerate(comp_errors(ps, os_)):
        assert e < TOL, (cgfd.COMPONENTS[c], e)
    for c, e in enumerate(comp_errors(valid(_fields(p)), valid(_fields(o)))):
        assert e < TOL, (cgfd.COMPONENTS[c], e)
    p.close()
    o.close()


def test_finite_fault_single_stages_match_fp64_oracle():
    """cgfd_rk_stage with explicit times (currT = 3): tW and W after 1..3 stages."""
    m = _fault_model()
    dirs = [(1, 1, -1), (-1, -1, 1), (1, 1, -1)]
    init = cases.random_fields(m, 5)
    for nst in (1, 2, 3):
        p = cgfd.Solver(m.desc(kernel=cgfd.KERNEL_FUSED))
        o = pyoracle.OracleSolver(m.desc(), 0)
        for s in (p, o):
            m.load(s)
            for c in range(9):
                s.set_field(c, init[c])
            for st in range(nst):
                s.rk_stage(st, 3, *dirs[st])
        for fset in (cgfd.SET_W, cgfd.SET_TW):
            for c, e in enumerate(comp_errors(valid(_fields(p, fset)), valid(_fields(o, fset)))):
                assert e < TOL, (nst, fset, cgfd.COMPONENTS[c], e)
        p.close()
        o.close()


def test_focal_points_in_a_batch_equal_single_runs():
    ms = models.batch_models(n=3, seed=11, nt=30, side=(28, 44), nabs_cells=5)
    ms[1] = models.with_finite_fault(ms[1], center=(3 + ms[1].ni // 2, 3 + ms[1].nj // 2,
                                                    3 + ms[1].nk - 8),
                                     length=5, width=3, m0=1e15, rise=0.08)
    steps = 24
    ref = []
    for m in ms:
        s = cgfd.Solver(m.desc())
        m.load(s)
        s.step(steps)
        ref.append((s.seismograms(), _fields(s)))
        s.close()
    b = cgfd.Batch([m.desc() for m in ms])
    for m, s in zip(ms, b.models):
        m.load(s)
    b.prepare()
    b.step(steps)
    b.sync()
    for q, s in enumerate(b.models):
        for e in comp_errors(s.seismograms(), ref[q][0]):
            assert e < TOL, q
        for e in comp_errors(valid(_fields(s)), valid(ref[q][1])):
            assert e < TOL, q
    b.close()


def test_focal_points_with_fp16_storage_follow_fp32():
    m = _fault_model()
    steps = 36
    out = {}
    for st in (cgfd.STORE_F32, cgfd.STORE_F16):
        s = cgfd.Solver(m.desc(storage=st))
        m.load(s)
        s.step(steps)
        out[st] = s.seismograms()[:, :, :steps]
        s.close()
    assert np.isfinite(out[cgfd.STORE_F16]).all()
    for e in comp_errors(out[cgfd.STORE_F16], out[cgfd.STORE_F32])[:3]:  # velocities
        assert e < 2e-2
