"""Point location and source smoothing on the host against fixtures made by
the reference's own source.cpp / common.cpp (tests/golden/make_source_golden.py,
its SrcSmooth and TypeDouble build): nearest-node location of forces,
moments and receivers (surface snapping above the hyper height), the
sub-cell shifts and the 7^3 Gaussian weights with the surface
renormalisation, and the source time functions.  Also the oracle's
spreading of smoothed sources on the CPU."""
import glob
import os

import numpy as np
import pytest

import cgfd
import models
import pyoracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(glob.glob(os.path.join(GOLDEN, "source_locate_*.npz")))
IDS = [os.path.basename(p)[:-4] for p in CASES]


def test_fixtures_present():
    assert len(CASES) == 2


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_location_matches_reference(path):
    g = np.load(path)
    x, y, z, hyp = g["x"], g["y"], g["z"], float(g["hyp"])
    for key in ("recv", "force", "moment"):
        pos = g[key + "_pos"]
        loc, posz = cgfd.locate_points(x, y, z, pos, hyp)
        if key == "recv":
            assert np.array_equal(loc, g["recv_loc"])
            # both branches: points above the hyper height snap to the surface
            above = pos[:, 2] > hyp
            assert above.any() and (~above).any()
            assert (loc[above, 2] == z.shape[2] - 4).all()
            assert np.array_equal(posz, g["recv_posz"])
        else:
            assert np.array_equal(posz, g[key + "_posz"])


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_smoothing_weights_match_reference(path):
    g = np.load(path)
    x, y, z, hyp = g["x"], g["y"], g["z"], float(g["hyp"])
    top = z.shape[2] - 4
    for kind, key in ((0, "force"), (1, "moment")):
        pos = g[key + "_pos"].copy()
        loc, posz = cgfd.locate_points(x, y, z, pos, hyp)
        pos[:, 2] = posz
        loc2, w = cgfd.source_smoothing(x, y, z, kind, pos, loc)
        assert np.array_equal(loc2, g[key + "_loc"])
        assert np.abs(w - g[key + "_w"]).max() <= 1e-14
        # blocks reaching above the surface are renormalised over the nodes
        # at or below it
        for q in range(len(loc)):
            kn = top + 1 - loc[q, 2] + 3
            if kn < 7:
                assert abs(w[q, :, :, :kn].sum() - 1.0) < 1e-12
            else:
                assert abs(w[q].sum() - 1.0) < 1e-12
        assert any(top + 1 - l[2] + 3 < 7 for l in loc)


def test_moment_shift_moves_a_node():
    """The curved case holds a moment point whose sub-cell search moves it
    to another node (MomentShiftPosition)."""
    g = np.load(os.path.join(GOLDEN, "source_locate_curved.npz"))
    pos = g["moment_pos"].copy()
    loc, posz = cgfd.locate_points(g["x"], g["y"], g["z"], pos, float(g["hyp"]))
    assert (loc != g["moment_loc"]).any()


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_source_time_functions_match_reference(path):
    g = np.load(path)
    nstf = 2 * (int(g["nt"]) + 1)
    s = cgfd.stf("Ricker", 0.0, 0.6, 2.0, nstf, float(g["stept"]) / 2.0)
    for key in ("force_stf", "moment_stf"):
        ref = g[key][0]
        assert np.abs(s - ref).max() <= 1e-6 * np.abs(ref).max()


def test_location_errors():
    g = np.load(CASES[0])
    x, y, z = g["x"], g["y"], g["z"]
    with pytest.raises(cgfd.CgfdError, match="outside the valid grid"):
        cgfd.source_smoothing(x, y, z, 1, np.zeros((1, 3)), np.array([[1, 5, 5]]))
    with pytest.raises(cgfd.CgfdError, match="bad smoothing"):
        cgfd.source_smoothing(x, y, z, 3, np.zeros((1, 3)), np.array([[5, 5, 5]]))


def _oracle_run(m, steps, smooth=None):
    o = pyoracle.OracleSolver(m.desc(), 0)
    m.load(o)
    for kind, w in (smooth or {}).items():
        o.set_source_smoothing(kind, w)
    o.step(steps)
    f = np.stack([o.get_field(c) for c in range(9)])
    s = o.seismograms()
    o.close()
    return f, s


def test_oracle_delta_weights_equal_point_sources():
    m = models.small_hill(nt=12, ni=20, nj=18, nk=16, force=True)
    d = np.zeros((1, 7, 7, 7))
    d[0, 3, 3, 3] = 1.0
    f0, s0 = _oracle_run(m, 8)
    f1, s1 = _oracle_run(m, 8, {0: d, 1: d})
    assert np.array_equal(f0, f1) and np.array_equal(s0, s1)


def test_oracle_spreading_conserves_the_moment():
    """One stage from rest: the stress RHS a smoothed moment source adds,
    times h^3 J, sums to the point source's whatever the weights (all its
    block inside the grid)."""
    m = models.small_flat(nt=12, ni=20, nj=18, nk=16)
    rng = np.random.default_rng(3)
    w = rng.uniform(0.0, 1.0, (1, 7, 7, 7))
    w /= w.sum()
    out = []
    for smooth in (None, {0: w}):
        o = pyoracle.OracleSolver(m.desc(), 0)
        m.load(o)
        if smooth:
            o.set_source_smoothing(0, w)
        o.rk_stage(0, 2, 1, 1, -1)
        out.append(np.stack([o.get_field(c, cgfd.SET_W) for c in range(3, 9)]))
        o.close()
    jac = m.metric["jac"]
    tot = [(a * jac[None]).sum(axis=(1, 2, 3)) for a in out]
    assert np.abs(out[0]).max() > 0
    assert np.allclose(tot[0], tot[1], rtol=1e-9, atol=0)
    assert np.count_nonzero(out[1][0]) > 300


def test_threaded_search_breaks_ties_in_scan_order():
    """Points exactly between nodes of a uniform grid (ties) and a search
    large enough to run on several threads: the node found is the first
    minimum in (i, j, k) order, as one sequential scan finds it."""
    ni, nj, nk, h = 40, 36, 30, 10.0
    i, j, k = np.meshgrid(np.arange(ni + 6), np.arange(nj + 6), np.arange(nk + 6), indexing="ij")
    x, y, z = i * h, j * h, (k - (nk + 2)) * h
    rng = np.random.default_rng(5)
    base = rng.integers([4, 4, 4], [ni + 1, nj + 1, nk + 1], size=(240, 3)).astype(np.float64)
    pos = (base + rng.integers(0, 2, size=(240, 3)) * 0.5) * h  # half-way on some axes
    pos[:, 2] -= (nk + 2) * h
    loc, posz = cgfd.locate_points(x, y, z, pos, hyper_height=1e9)
    vx, vy, vz = (a[3:-3, 3:-3, 3:-3].ravel() for a in (x, y, z))
    for q in range(len(pos)):
        d = (vx - pos[q, 0]) ** 2 + (vy - pos[q, 1]) ** 2 + (vz - pos[q, 2]) ** 2
        t = int(np.argmin(d))  # first minimum in C (i, j, k) order
        want = np.array(np.unravel_index(t, (ni, nj, nk))) + 3
        assert np.array_equal(loc[q], want), q
    assert np.array_equal(posz, pos[:, 2])


WAVELET_NAMES = ("Gauss", "gauss", "Ricker", "ricker", "Bell", "bell", "BELL", "Step")


@pytest.mark.parametrize("name", WAVELET_NAMES)
def test_wavelets_match_reference(name):
    """cgfd_stf (FP32 out) and the oracle's (FP64) against the reference's
    cal_stf_force / cal_stf_moment samples of every wavelet type, at start
    times 0 and 0.05 s (tests/golden/source_wavelets.npz)."""
    g = np.load(os.path.join(GOLDEN, "source_wavelets.npz"))
    n, dt = 2 * (int(g["nt"]) + 1), float(g["stept"]) / 2.0
    t0, f0 = (float(v) for v in g["t0f0_" + name])
    for start in (0.0, 0.05):
        got32 = cgfd.stf(name, start, t0, f0, n, dt)
        got64 = pyoracle.stf(cgfd.STF_TYPES[name], start, t0, f0, n, dt)
        for kind in ("force", "moment"):
            ref = g[f"{kind}_{name}_{start:g}"]
            scale = np.abs(ref).max()
            assert scale > 0
            assert np.abs(got32 - ref).max() <= 1e-6 * scale, (kind, start)
            assert np.abs(got64 - ref).max() <= 1e-12 * scale, (kind, start)


def test_angle2moment_matches_reference():
    """Strike/dip/rake to a moment tensor as the reference's source::
    angle2moment, times mu at the source as its cal_index applies it."""
    g = np.load(os.path.join(GOLDEN, "source_wavelets.npz"))
    mu = float(g["mu"])
    for fn in (cgfd.angle2moment, pyoracle.angle2moment):
        m6 = np.array([fn(*a) for a in g["angles"]]) * mu
        assert np.abs(m6 - g["m6"]).max() <= 1e-12 * np.abs(g["m6"]).max()
