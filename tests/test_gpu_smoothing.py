"""Smoothed sources on the GPU (cgfd_set_source_smoothing): moments, forces
and focal points spread over their 7^3 blocks as the reference's SrcSmooth
build of LoadMoment / LoadForce / LoadRmom does.  Against the FP64 oracle
within the 1e-5 parity bar (kernel families, whole steps and single stages,
blocks cut by the grid's sides and its surface); with one-node weights equal
to the point sources; off again after a new upload; in a batch as alone;
with FP16 storage close to FP32."""
import dataclasses
import os

import numpy as np
import pytest

import cases
import cgfd
import models
import pyoracle
from helpers import comp_errors, valid

pytestmark = pytest.mark.gpu

TOL = 1e-5
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _model(nt=40):
    """small_hill with a surface force and a second moment next to the
    x- side (its block crosses the side; the force's crosses the surface)."""
    m = models.small_hill(nt=nt, force=True)
    loc = np.concatenate([m.mnt_loc, [[4, 3 + m.nj // 3, 3 + m.nk - 6]]]).astype(np.int32)
    m6 = np.concatenate([m.mnt_m6, 0.5 * m.mnt_m6[:, ::-1]]).astype(np.float32)
    stf = np.concatenate([m.mnt_stf, m.mnt_stf]).astype(np.float32)
    return dataclasses.replace(m, mnt_loc=loc, mnt_m6=m6, mnt_stf=stf)


def _weights(n, seed):
    """A Gaussian block of the reference's (from the location fixtures),
    then random positive blocks normalised to 1."""
    g = np.load(os.path.join(GOLDEN, "source_locate_hill.npz"))
    rng = np.random.default_rng(seed)
    w = rng.uniform(0.0, 1.0, (n, 7, 7, 7))
    w /= w.sum(axis=(1, 2, 3), keepdims=True)
    w[0] = g["moment_w"][0]
    return w


def _fields(s, fset=0):
    return np.stack([s.get_field(c, fset) for c in range(9)])


def _run(solver, m, steps, smooth):
    m.load(solver)
    for kind, w in smooth.items():
        solver.set_source_smoothing(kind, w)
    solver.step(steps)
    return solver.seismograms()[:, :, :steps], _fields(solver)


@pytest.mark.parametrize("kernel", [cgfd.KERNEL_SIMPLE, cgfd.KERNEL_FUSED, cgfd.KERNEL_SCALAR],
                         ids=["simple", "fused", "scalar"])
def test_smoothed_point_sources_match_fp64_oracle(kernel):
    m = _model()
    smooth = {0: _weights(len(m.mnt_loc), 1), 1: _weights(len(m.frc_loc), 2)}
    steps = 36
    p = cgfd.Solver(m.desc(kernel=kernel))
    ps, pf = _run(p, m, steps, smooth)
    o = pyoracle.OracleSolver(m.desc(), 0)
    os_, of = _run(o, m, steps, smooth)
    assert np.abs(os_[:3]).max() > 0
    for c, e in enumerate(comp_errors(ps, os_)):
        assert e < TOL, (cgfd.COMPONENTS[c], e)
    for c, e in enumerate(comp_errors(valid(pf), valid(of))):
        assert e < TOL, (cgfd.COMPONENTS[c], e)
    p.close()
    o.close()


def test_smoothed_sources_single_stages_match_fp64_oracle():
    """cgfd_rk_stage with explicit times (currT = 3): W and tW after 1..3 stages."""
    m = _model()
    smooth = {0: _weights(len(m.mnt_loc), 3), 1: _weights(len(m.frc_loc), 4)}
    dirs = [(1, 1, -1), (-1, -1, 1), (1, 1, -1)]
    init = cases.random_fields(m, 5)
    for nst in (1, 2, 3):
        p = cgfd.Solver(m.desc(kernel=cgfd.KERNEL_FUSED))
        o = pyoracle.OracleSolver(m.desc(), 0)
        for s in (p, o):
            m.load(s)
            for kind, w in smooth.items():
                s.set_source_smoothing(kind, w)
            for c in range(9):
                s.set_field(c, init[c])
            for st in range(nst):
                s.rk_stage(st, 3, *dirs[st])
        for fset in (cgfd.SET_W, cgfd.SET_TW):
            for c, e in enumerate(comp_errors(valid(_fields(p, fset)), valid(_fields(o, fset)))):
                assert e < TOL, (nst, fset, cgfd.COMPONENTS[c], e)
        p.close()
        o.close()


def test_smoothed_focal_points_match_fp64_oracle():
    m = models.small_hill(nt=40, nabs=(5, 6, 4, 5, 5, 0))
    m = dataclasses.replace(m, mnt_loc=np.zeros((0, 3), np.int32),
                            mnt_m6=np.zeros((0, 6), np.float32),
                            mnt_stf=np.zeros((0, m.mnt_stf.shape[1]), np.float32))
    m = models.with_finite_fault(m, center=(3 + m.ni // 2, 3 + m.nj // 2, 3 + m.nk - 9),
                                 length=6, width=4, m0=1e15, vr=2500.0, rise=0.06)
    smooth = {2: _weights(len(m.foc_loc), 5)}
    steps = 36
    p = cgfd.Solver(m.desc(kernel=cgfd.KERNEL_FUSED))
    ps, pf = _run(p, m, steps, smooth)
    o = pyoracle.OracleSolver(m.desc(), 0)
    os_, of = _run(o, m, steps, smooth)
    assert np.abs(os_[:3]).max() > 0
    for c, e in enumerate(comp_errors(ps, os_)):
        assert e < TOL, (cgfd.COMPONENTS[c], e)
    for c, e in enumerate(comp_errors(valid(pf), valid(of))):
        assert e < TOL, (cgfd.COMPONENTS[c], e)
    p.close()
    o.close()


def test_one_node_weights_equal_point_sources_and_reupload_turns_off():
    m = _model(nt=30)
    steps = 24
    d = np.zeros((len(m.mnt_loc), 7, 7, 7))
    d[:, 3, 3, 3] = 1.0
    df = np.zeros((len(m.frc_loc), 7, 7, 7))
    df[:, 3, 3, 3] = 1.0
    base = _run(cgfd.Solver(m.desc()), m, steps, {})
    one = _run(cgfd.Solver(m.desc()), m, steps, {0: d, 1: df})
    for a, b in zip(base, one):
        assert np.abs(a - b).max() <= 1e-6 * np.abs(a).max()
    # weights set, then the sources uploaded again: point sources once more
    s = cgfd.Solver(m.desc())
    m.load(s)
    s.set_source_smoothing(0, _weights(len(m.mnt_loc), 6))
    s.upload_moments(m.mnt_loc, m.mnt_m6, m.mnt_stf)
    s.step(steps)
    assert np.array_equal(s.seismograms()[:, :, :steps], base[0])
    s.close()


def test_smoothing_checks():
    m = _model(nt=10)
    s = cgfd.Solver(m.desc())
    m.load(s)
    with pytest.raises(cgfd.CgfdError, match="differs"):
        s.set_source_smoothing(0, _weights(len(m.mnt_loc) + 1, 1))
    with pytest.raises(cgfd.CgfdError, match="kind"):
        s.set_source_smoothing(3, _weights(1, 1))
    s.close()


def test_smoothed_sources_in_a_batch_equal_single_runs():
    ms = models.batch_models(n=3, seed=3, nt=30, side=(28, 44), nabs_cells=5)
    ms[1] = dataclasses.replace(ms[1], mnt_smooth=_weights(len(ms[1].mnt_loc), 7))
    ms[2] = models.with_finite_fault(ms[2], center=(3 + ms[2].ni // 2, 3 + ms[2].nj // 2,
                                                    3 + ms[2].nk - 8),
                                     length=5, width=3, m0=1e15, rise=0.08)
    ms[2] = dataclasses.replace(ms[2], foc_smooth=_weights(len(ms[2].foc_loc), 8))
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


def test_smoothed_sources_with_fp16_storage_follow_fp32():
    m = _model()
    smooth = {0: _weights(len(m.mnt_loc), 9), 1: _weights(len(m.frc_loc), 10)}
    steps = 36
    out = {}
    for st in (cgfd.STORE_F32, cgfd.STORE_F16):
        s = cgfd.Solver(m.desc(storage=st))
        out[st] = _run(s, m, steps, smooth)[0]
        s.close()
    assert np.isfinite(out[cgfd.STORE_F16]).all()
    for e in comp_errors(out[cgfd.STORE_F16], out[cgfd.STORE_F32])[:3]:  # velocities
        assert e < 2e-2
