"""Host pre-processing (FP64): the library's metric, CFS-PML, STF and
moment-tensor helpers against the oracle's restatement of
gridmesh::calmetric, absorb::CalCFSfactors, mathfunc wavelets and
source::angle2moment."""
import numpy as np
import pytest

import cgfd
import models
import pyoracle


def test_metric_matches_oracle_on_curved_grid():
    ni, nj, nk, h = 14, 12, 16, 100.0
    x, y, z = models._coords(ni, nj, nk, h, 60.0, 120.0, 400.0, 600.0, 10)
    a = cgfd.metric_from_coords(ni, nj, nk, h, x, y, z)
    b = pyoracle.metric_from_coords(ni, nj, nk, h, x, y, z)
    for k in a:
        np.testing.assert_allclose(a[k], b[k], rtol=1e-12, atol=1e-14, err_msg=k)
    v = (slice(3, -3),) * 3
    assert np.abs(a["zeta_x"][v]).max() > 1e-3  # really curved
    assert np.all(a["jac"][v] > 0)


def test_flat_grid_has_trivial_metric():
    ni, nj, nk, h = 10, 9, 8, 50.0
    x, y, z = models._coords(ni, nj, nk, h, h, h, 0.0, 1.0, 5)
    m = cgfd.metric_from_coords(ni, nj, nk, h, x, y, z)
    v = (slice(3, -3),) * 3
    assert np.all(m["zeta_x"][v] == 0) and np.all(m["zeta_y"][v] == 0)
    assert np.all(m["zeta_z"][v] == 1) and np.all(m["jac"][v] == 1)
    assert np.all(m["xi_x"][v] == 1) and np.all(m["eta_y"][v] == 1)


@pytest.mark.parametrize("nabs", [(31, 0, 0, 0, 0, 0), (0, 0, 0, 28, 0, 0), (0, 0, 0, 0, -1, 0)])
def test_cfs_factors_refuse_layers_wider_than_the_grid(nabs):
    """A layer wider than the grid along its axis (or of negative width) is
    an argument error, not a write before or past the profile arrays."""
    ni, nj, nk = 30, 27, 25
    dl = [np.full(n + 6, 100.0) for n in (ni, nj, nk)]
    with pytest.raises(cgfd.CgfdError, match="wider than the grid"):
        cgfd.cfs_factors(ni, nj, nk, nabs, [8500.0] * 6, [2.5] * 6, [5.0] * 6, *dl)


@pytest.mark.parametrize("nabs", [(12, 12, 12, 12, 12, 0), (3, 5, 0, 7, 4, 0), (6, 4, 5, 5, 5, 0)])
def test_cfs_factors_match_oracle(nabs):
    ni, nj, nk = 30, 27, 25
    rng = np.random.default_rng(3)
    dl = [rng.uniform(40, 160, n + 6) for n in (ni, nj, nk)]
    vel, bm, am = [8500.0] * 6, [2.5] * 6, [5.0] * 6
    a = cgfd.cfs_factors(ni, nj, nk, nabs, vel, bm, am, *dl)
    b = pyoracle.cfs_factors(ni, nj, nk, nabs, vel, bm, am, *dl)
    for ga, gb in zip(a, b):
        for xa, xb in zip(ga, gb):
            np.testing.assert_allclose(xa, xb, rtol=1e-13, atol=0)
    apd, B, DB = a
    # interior: no stretching, no damping
    assert B[0][3 + nabs[0]] == 1.0 and DB[0][3 + nabs[0]] == 0.0
    # damping grows outwards in the X1 layer
    if nabs[0] > 1:
        assert DB[0][3] > DB[0][3 + nabs[0] - 1] > 0


def test_cfs_profile_values_for_uniform_spacing():
    # L = (w - c) * h for the c-th cell from the outer edge; d = dmax (L/L0)^2
    ni, nj, nk, w, h = 30, 30, 30, 10, 100.0
    dl = [np.full(n + 6, h) for n in (ni, nj, nk)]
    apd, B, DB = cgfd.cfs_factors(ni, nj, nk, (w, w, w, w, w, 0), [6000.0] * 6,
                                  [2.0] * 6, [3.0] * 6, *dl)
    R = 10 ** (-(np.log10(w) - 1) / np.log10(2) - 3)
    L0 = w * h
    dmax = -6000.0 / 2 / L0 * np.log(R) * 3
    r = (w - np.arange(w)) / w
    np.testing.assert_allclose(B[0][3:3 + w], 1 + (2.0 - 1) * r ** 2, rtol=1e-14)
    np.testing.assert_allclose(DB[0][3:3 + w], dmax * r ** 2 / (1 + r ** 2), rtol=1e-14)
    np.testing.assert_allclose(apd[0][3:3 + w], 3.0 * (1 - r) + dmax * r ** 2 / (1 + r ** 2), rtol=1e-14)
    assert np.all(B[2][nk + 3 - 3:] == 1.0)  # no layer at the top


@pytest.mark.parametrize("kind", ["Gauss", "gauss", "Ricker", "ricker", "Bell", "bell", "BELL", "Step"])
def test_stf_matches_oracle(kind):
    a = cgfd.stf(kind, 0.1, 0.6, 2.0 if "icker" in kind else 0.3, 1002, 0.004)
    b = pyoracle.stf(cgfd.STF_TYPES[kind], 0.1, 0.6, 2.0 if "icker" in kind else 0.3, 1002, 0.004)
    np.testing.assert_allclose(a, b.astype(np.float32), rtol=1e-6, atol=1e-12 * np.abs(b).max())
    assert np.abs(a).max() > 0


def test_angle2moment_matches_oracle_and_is_traceless():
    for sdr in [(30, 60, 90), (0, 90, 0), (137.5, 22.0, -45.0)]:
        a = cgfd.angle2moment(*sdr)
        b = pyoracle.angle2moment(*sdr)
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-15)
        assert abs(a[0] + a[1] + a[2]) < 1e-15
