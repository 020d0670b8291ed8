"""The CPU oracle against golden vectors produced by the reference's own CUDA
device runtime on a B200 (tests/golden/make_golden.py).  This pins the
oracle: seismograms and stage outputs within 1e-5 relative L2 (the reference
computes in FP32, the oracle in FP64)."""
import glob
import os

import numpy as np
import pytest

import cases
from helpers import comp_errors, rel_l2

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-5


def _golden_names():
    # the stepping fixtures of the reference's runtime (the vmap-grid, source,
    # output and par-file fixtures and the FP64 oracle's c1_fp64_* have their
    # own tests)
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith(("grid_vmap_", "source_", "outputs_",
                                                         "parfiles_", "c1_fp64_")))


def test_golden_set_is_complete():
    assert set(_golden_names()) == set(cases.CASES), "regenerate tests/golden (make_golden.py)"


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_oracle_matches_reference_golden(name):
    path = os.path.join(GOLDEN, f"{name}.npz")
    if not os.path.exists(path):
        pytest.fail(f"missing golden file {path}")
    g = np.load(path)
    m, nsteps, nstages, init = cases.build(name)
    assert str(g["digest"]) == cases.model_digest(m, init), "inputs changed since the golden run"
    seis, fw, w = cases.run_oracle(m, nsteps, nstages, init)
    if nsteps:
        for c in range(3):  # velocity seismograms, strictly per component
            assert rel_l2(seis[c], g["seis"][c]) < TOL
        for c, e in enumerate(comp_errors(seis, g["seis"])):
            assert e < TOL, (c, e)
    if nstages:
        wv = w[:, 3:-3, 3:-3, 3:-3]
        for c, e in enumerate(comp_errors(wv, g["w"])):
            assert e < TOL, (c, e)


def test_oracle_fp32_and_fp64_agree():
    m, nsteps, nstages, init = cases.build("hill_60")
    a = cases.run_oracle(m, nsteps, nstages, init, prec=0)[0]
    b = cases.run_oracle(m, nsteps, nstages, init, prec=1)[0]
    for e in comp_errors(b, a):
        assert e < 1e-5


def test_oracle_matches_reference_focal_pv_snapshot_golden():
    """The reference's finite fault (InterpFocus / LoadRmom), peak velocity
    (IterationFinalPV) and snapshots (SWpick) against the oracle's."""
    path = os.path.join(GOLDEN, f"{cases.OUTPUT_CASE}.npz")
    if not os.path.exists(path):
        pytest.fail(f"missing golden file {path}")
    g = np.load(path)
    m = cases.build_outputs_case()
    assert str(g["digest"]) == cases.model_digest(m), "inputs changed since the golden run"
    assert np.array_equal(g["snap_points"], cases.snap_points())
    seis, pv, snap = cases.run_oracle_outputs(m, int(g["nsteps"]))
    assert np.abs(g["seis"][:3]).max() > 0 and g["pv"].max() > 0
    for c in range(3):
        assert rel_l2(seis[c], g["seis"][c]) < TOL, c
        assert rel_l2(pv[c], g["pv"][c]) < TOL, c
    for c, e in enumerate(comp_errors(seis, g["seis"])):
        assert e < TOL, (c, e)
    for c, e in enumerate(comp_errors(snap, g["snap"])):
        assert e < TOL, (c, e)
