"""The finite-fault source, peak ground velocity and snapshots against the
reference's own runtime (oracle/_ref/ref_wavesim) on the same inputs:

  * focal points: the reference interpolates each point's moment-rate series
    on the host every stage (InterpFocus / ExtractValue, src/calculate.cu:
    1421-1428, 2586-2676) and injects them with LoadRmom (6257-6328); the
    solver interpolates and injects on the device (cgfd_upload_focal);
  * peak velocity: the reference's last stage keeps max |V| of the top valid
    layer (IterationFinalPV, 6736-6851; SynPV 1709); the solver's step graph
    does the same (cgfd_enable_peak_velocity / cgfd_get_peak_velocity);
  * snapshots: the reference copies FW at its snapshot points after every
    tinv-th step (C2DSnapPick / SWpick, 2230-2445); the solver gathers a
    strided sub-volume (cgfd_get_snapshot).

One run of tests/cases.py's OUTPUT_CASE, live against the reference and
against the golden file it wrote, within the 1e-5 parity bar.
"""
import os

import numpy as np
import pytest

import cases
import cgfd
import refio
from helpers import comp_errors, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                      f"{cases.OUTPUT_CASE}.npz")


def _run_product(m, nsteps):
    s = cgfd.Solver(m.desc())
    m.load(s)
    s.enable_peak_velocity(True)
    ntime = (m.nt + cases.SNAP_TINV - 1) // cases.SNAP_TINV
    snap = np.zeros((9, len(cases.snap_points()), ntime), np.float32)
    for t in range(nsteps):
        s.step(1)
        if t % cases.SNAP_TINV == 0:
            v = s.snapshot(cases.SNAP_START, cases.SNAP_COUNT, cases.SNAP_STRIDE)
            snap[:, :, t // cases.SNAP_TINV] = v.reshape(9, -1)
    out = s.seismograms(), s.peak_velocity(), snap
    s.close()
    return out


def _compare(seis, pv, snap, ref_seis, ref_pv, ref_snap, what):
    assert np.abs(ref_seis[:3]).max() > 0 and ref_pv.max() > 0, what
    for c in range(3):
        e = rel_l2(seis[c], ref_seis[c])
        assert e < TOL, f"{what}: seismogram {cgfd.COMPONENTS[c]} {e:.3e}"
        e = rel_l2(pv[c], ref_pv[c])
        assert e < TOL, f"{what}: peak velocity {cgfd.COMPONENTS[c]} {e:.3e}"
    for c, e in enumerate(comp_errors(seis, ref_seis)):
        assert e < TOL, f"{what}: seismogram {cgfd.COMPONENTS[c]} {e:.3e}"
    for c, e in enumerate(comp_errors(snap, ref_snap)):
        assert e < TOL, f"{what}: snapshot {cgfd.COMPONENTS[c]} {e:.3e}"


def test_focal_peak_velocity_and_snapshots_match_reference():
    m = cases.build_outputs_case()
    pts = cases.snap_points()
    r = refio.run(m, m.nt, fields=False, focal=True, peak_velocity=True, snap_points=pts,
                  snap_tinv=cases.SNAP_TINV)
    seis, pv, snap = _run_product(m, m.nt)
    _compare(seis, pv, snap, r["seis"], r["pv"][:, 3:-3, 3:-3], r["snap"], "live reference")


def test_focal_peak_velocity_and_snapshots_match_golden():
    g = np.load(GOLDEN)
    m = cases.build_outputs_case()
    assert str(g["digest"]) == cases.model_digest(m)
    seis, pv, snap = _run_product(m, int(g["nsteps"]))
    _compare(seis, pv, snap, g["seis"], g["pv"], g["snap"], "golden")
