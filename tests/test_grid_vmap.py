"""cgfd_grid_vmap (the vmap grid generation of the reference's gridmesh)
against fixtures made by the reference's own gridmesh.cpp
(tests/golden/make_grid_golden.py): graded layers on both branches of its
spacing search, hybrid grids with and without a graded layer; node
coordinates including the extrapolated ghost nodes and ConIndex, and the
metric of each grid against the reference's calmetric (with its mirrored
ghost nodes), and the ADE CFS-PML profiles on that metric against its
absorb::CalCFSfactors.  Also the reference's input checks."""
import glob
import os

import numpy as np
import pytest

import cgfd
import pyoracle

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


METRIC = ("xi_x", "xi_y", "xi_z", "eta_x", "eta_y", "eta_z", "zeta_x", "zeta_y", "zeta_z", "jac")


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[:-4] for p in CASES])
def test_metric_matches_reference_calmetric(path):
    """cgfd_metric_from_coords and the oracle's restatement against the
    reference's gridmesh::calmetric on the reference's own grid (steph 100):
    all ten arrays, ghost nodes included, to 1e-12 of each array's scale
    (equal in practice)."""
    g = np.load(path)
    ni, nj, nk = int(g["ni"]), int(g["nj"]), int(g["nk"])
    for fn in (cgfd.metric_from_coords, pyoracle.metric_from_coords):
        m = fn(ni, nj, nk, 100.0, g["x"], g["y"], g["z"])
        for q, name in enumerate(METRIC):
            ref = g["metric"][q]
            scale = max(np.abs(ref).max(), 1e-300)
            assert np.abs(m[name] - ref).max() <= 1e-12 * scale, (fn.__module__, name)


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[:-4] for p in CASES])
def test_cfs_factors_match_reference(path):
    """cgfd_cfs_factors and the oracle's restatement against the reference's
    absorb::CalCFSfactors on the reference's grid and metric: APD, B and DB
    along x, y and z (layer thicknesses steph/|grad xi| at (i, 3, 3), and
    likewise for eta and zeta, as the reference measures them)."""
    g = np.load(path)
    ni, nj, nk, h = int(g["ni"]), int(g["nj"]), int(g["nk"]), 100.0
    m = dict(zip(METRIC, g["metric"]))

    def thickness(a, b, c):
        n = np.sqrt(a * a + b * b + c * c)
        return np.where(n > 0, h / np.where(n > 0, n, 1.0), 0.0)

    dl = (thickness(m["xi_x"][:, 3, 3], m["xi_y"][:, 3, 3], m["xi_z"][:, 3, 3]),
          thickness(m["eta_x"][3, :, 3], m["eta_y"][3, :, 3], m["eta_z"][3, :, 3]),
          thickness(m["zeta_x"][3, 3, :], m["zeta_y"][3, 3, :], m["zeta_z"][3, 3, :]))
    nabs = tuple(int(v) for v in g["pml_nabs"])
    args = (ni, nj, nk, nabs, [float(g["pml_velabs"])] * 6, [float(g["pml_bmax"])] * 6,
            [float(g["pml_amax"])] * 6, *dl)
    for fn in (cgfd.cfs_factors, pyoracle.cfs_factors):
        apd, b, db = fn(*args)
        for ax, key in enumerate(("pml_x", "pml_y", "pml_z")):
            ref = g[key]
            for q, got in enumerate((apd[ax], b[ax], db[ax])):
                scale = max(np.abs(ref[q]).max(), 1e-300)
                assert np.abs(np.asarray(got) - ref[q]).max() <= 1e-12 * scale, (fn.__module__, key, q)
        assert np.abs(np.asarray(db[0])).max() > 0 and np.abs(np.asarray(db[2])).max() > 0
