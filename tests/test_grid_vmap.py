"""cgfd_grid_vmap (the vmap grid generation of the reference's gridmesh)
against fixtures made by the reference's own gridmesh.cpp
(tests/golden/make_grid_golden.py): graded layers on both branches of its
spacing search, hybrid grids with and without a graded layer; node
coordinates including the extrapolated ghost nodes and ConIndex.  Also the
reference's input checks."""
import glob
import os

import numpy as np
import pytest

import cgfd

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(glob.glob(os.path.join(GOLDEN, "grid_vmap_*.npz")))


def test_fixtures_present():
    assert len(CASES) == 4


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[:-4] for p in CASES])
def test_grid_matches_reference_gridmesh(path):
    g = np.load(path)
    x, y, z, con = cgfd.grid_vmap(int(g["ni"]), int(g["nj"]), int(g["nk"]), g["gridpoints"],
                                  g["equalspacing"], g["anchor"], bool(g["hybrid"]),
                                  float(g["depth"]))
    assert con == int(g["con_index"])
    scale = np.abs(g["z"]).max()
    for got, ref in ((x, g["x"]), (y, g["y"]), (z, g["z"])):
        assert np.abs(got - ref).max() <= 1e-12 * scale


def test_grid_checks_follow_the_reference():
    g = np.load(CASES[0])
    ni, nj, nk = int(g["ni"]), int(g["nj"]), int(g["nk"])
    gp, eq, a = g["gridpoints"], g["equalspacing"], g["anchor"]
    with pytest.raises(cgfd.CgfdError, match="intervals"):
        cgfd.grid_vmap(ni, nj, nk + 1, gp, eq, a)
    with pytest.raises(cgfd.CgfdError, match="first and the last"):
        cgfd.grid_vmap(ni, nj, nk, gp, [0, 1, 1], a)
    bad = a.copy()
    bad[2, 3, 3] = bad[2, 3, 2] + 1.0  # an interface above the one over it
    with pytest.raises(cgfd.CgfdError, match="decrease"):
        cgfd.grid_vmap(ni, nj, nk, gp, eq, bad)
    with pytest.raises(cgfd.CgfdError, match="conversion depth"):
        cgfd.grid_vmap(ni, nj, nk, gp, eq, a, hybrid=True, convers_depth=-1e6)
