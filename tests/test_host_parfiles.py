"""The host program wavesim_b200 on the reference's par files (no GPU: its
--dump mode stops before creating a solver).

Pinned on the reference: the vmap grid it reads and generates, the metric
and the CFS-PML profiles equal the reference's own gridmesh reader,
calmetric and CalCFSfactors on the same files (tests/golden/
parfiles_ref_grid.npz, from oracle/_ref/ref_grid; make_parfiles.py).  The
rest of the par-file semantics -- distance2meter, the hyper heights, the
strike/dip/rake moments times mu at the source node, the wavelets, receiver
lines, the volume media file -- against the library's own entry points
(each pinned on the reference elsewhere) called on the values the par files
hold.
"""
import os

import numpy as np
import pytest

import cgfd
import hostio

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def dump(tmp_path_factory):
    if not os.path.exists(hostio.HOST):
        pytest.fail(f"{hostio.HOST} is not built (make -C copara-cgfd3d_b200)")
    d = str(tmp_path_factory.mktemp("par"))
    hostio.copy_parfiles(d)
    hostio.run(d, "--dump", "model.bin")
    return hostio.read_dump(os.path.join(d, "model.bin"))


def _close(a, b, rtol=1e-12):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() <= rtol * scale


def test_grid_metric_and_pml_equal_the_references_own(dump):
    g = np.load(os.path.join(GOLDEN, "parfiles_ref_grid.npz"))
    assert dump["con"] == int(g["con"])
    for k in ("x", "y", "z", "zeta_x", "zeta_y", "zeta_z", "jac"):
        assert _close(dump[k], g[k]), k
    names = ("apd_x", "apd_y", "apd_z", "b_x", "b_y", "b_z", "db_x", "db_y", "db_z")
    for q, k in enumerate(names):
        assert _close(dump["pml"][q], g[k]), k
    assert dump["nabs"] == (6, 6, 6, 6, 6, 0)


def test_media_from_the_classic_volume_file(dump):
    from scipy.io import netcdf_file
    with netcdf_file(os.path.join(hostio.PARFILES, "media_volume.nc"), "r", mmap=False) as f:
        ax = [np.array(f.variables[n][:], np.float64) for n in ("x", "y", "depth")]
        vol = [np.array(f.variables[n][:], np.float32) for n in ("Vp", "Vs", "rho")]
    a, b, r = cgfd.media_volume(dump["x"], dump["y"], dump["z"], *ax, *vol, 100.0, 0.1)
    assert np.array_equal(dump["alpha"], a) and np.array_equal(dump["beta"], b)
    assert np.array_equal(dump["rho"], r)
    v = (slice(3, -3),) * 3
    assert dump["alpha"][v].min() >= 3200.0 and dump["alpha"][v].max() <= 5700.0


def test_sources_follow_source_dat(dump):
    import make_parfiles as mp
    x, y, z = dump["x"], dump["y"], dump["z"]
    nstf = 2 * (dump["nt"] + 1)
    # the force: km -> m, located with source_hyper_height * distance2meter
    fr = np.array(mp.FORCES)
    loc, _ = cgfd.locate_points(x, y, z, fr[:, :3] * 1e3, 9.0 * 1e3)
    assert np.array_equal(dump["floc"], loc)
    assert np.array_equal(dump["f3"], (fr[:, 5:8] * fr[:, 4:5]).astype(np.float32))
    w = cgfd.stf(mp.FORCE_STF[0], fr[0, 3], mp.FORCE_STF[1], mp.FORCE_STF[2], nstf,
                 dump["stept"] / 2)
    assert np.array_equal(dump["fstf"][0], w)
    # moments given as strike/dip/rake: x m0 x mu at the node
    mr = np.array(mp.MOMENTS)
    loc, _ = cgfd.locate_points(x, y, z, mr[:, :3] * 1e3, 9.0 * 1e3)
    assert np.array_equal(dump["mloc"], loc)
    for q in range(len(mr)):
        i, j, k = loc[q]
        mu = np.float32(dump["rho"][i, j, k]) * dump["beta"][i, j, k] * dump["beta"][i, j, k]
        m6 = (cgfd.angle2moment(*mr[q, 5:8]) * mr[q, 4]).astype(np.float32) * np.float32(mu)
        assert np.allclose(dump["m6"][q], m6, rtol=2e-7, atol=0), q
        w = cgfd.stf(mp.MOMENT_STF[0], mr[q, 3], mp.MOMENT_STF[1], mp.MOMENT_STF[2], nstf,
                     dump["stept"] / 2)
        assert np.array_equal(dump["mstf"][q], w)
    assert dump["nfoc"] == 0


def test_receivers_and_lines_follow_station_dat(dump):
    import make_parfiles as mp
    pts = [r for r in mp.RECV]
    for p0, dp, n in mp.LINES:
        pts += [tuple(p0[a] + j * dp[a] for a in range(3)) for j in range(n)]
    loc, posz = cgfd.locate_points(dump["x"], dump["y"], dump["z"], np.array(pts), 8000.0e3)
    assert np.array_equal(dump["rloc"], loc)
    assert np.allclose(dump["rpos"][:, 2], posz.astype(np.float32))
    top = dump["nk"] + 2
    assert loc[0, 2] == top and loc[2, 2] < top  # snapped to the surface / at depth


def test_host_reports_bad_par_files(tmp_path):
    d = str(tmp_path)
    hostio.copy_parfiles(d)
    conf = os.path.join(d, "SeisFD3D.conf")
    txt = open(conf).read()
    open(conf, "w").write(txt.replace("grid_type = vmap", "grid_type = point"))
    with pytest.raises(RuntimeError, match="only vmap grids"):
        hostio.run(d, "--dump", "m.bin")
    open(conf, "w").write(txt.replace("absorb_filename = absorb.dat", "absorb_filename = no.dat"))
    with pytest.raises(RuntimeError, match="cannot open"):
        hostio.run(d, "--dump", "m.bin")


@pytest.mark.parametrize("fname,old,new,match", [
    ("source.dat", "number_of_force_source = 1", "number_of_force_source = 2147483647",
     "out of range"),
    ("source.dat", "number_of_moment_source = 2", "number_of_moment_source = 3",
     "moment block too short"),
    ("station.dat", "snap_002 = 24 1 1 1 20 16 1 2 2 20 3", "snap_002 = 24 1 1 1 21 16 1 2 2 20 3",
     "inside the grid"),
    ("station.dat", "line_001 = -1500 0 9e+06 | 500 0 0 | 7",
     "line_001 = -1500 0 9e+06 | 500 0 0 | 1e12", "receiver count out of range"),
    ("SeisFD3D.conf", "nj    = 40", "nj    = 2147483647", "out of range"),
    ("grid_vmap.dat", "-2350.000000 -1950.000000 0.318052 -3100.000000",
     "-2350.000000 -1950.000000 nan -3100.000000", "anchor values must be finite"),
])
def test_host_bounds_what_par_files_ask_for(tmp_path, fname, old, new, match):
    """Counts and ranges read from the par files are checked before they size
    an allocation or an index: source and receiver counts, the anchor blocks'
    lengths, snapshot windows (start + (count - 1) * stride inside the grid),
    the grid's dimensions and the vmap anchors (finite)."""
    d = str(tmp_path)
    hostio.copy_parfiles(d)
    p = os.path.join(d, fname)
    txt = open(p).read()
    assert old in txt
    open(p, "w").write(txt.replace(old, new))
    with pytest.raises(RuntimeError, match=match):
        hostio.run(d, "--dump", "m.bin")
