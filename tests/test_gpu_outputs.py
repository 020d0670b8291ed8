"""Outputs beside the seismograms: peak ground velocity, sub-volume
snapshots, and the reference's seismo.nc / peakvel.nc variables written as
NetCDF classic files (read back here with scipy's independent reader)."""
import numpy as np
import pytest

import cgfd
import models

pytestmark = pytest.mark.gpu


def _run(steps=30, pgv=False):
    m = models.small_hill(nt=40)
    s = cgfd.Solver(m.desc())
    m.load(s)
    if pgv:
        s.enable_peak_velocity(True)
    s.step(steps)
    return m, s


def test_peak_velocity_is_the_max_of_the_surface_seismograms():
    m, s = _run(pgv=True)
    pv = s.peak_velocity()
    seis = s.seismograms()[:, :, :30]
    top = m.nk + 2
    for r, (i, j, k) in enumerate(m.rcv_loc):
        assert k == top
        for c in range(3):
            assert pv[c, i - 3, j - 3] == np.abs(seis[c, r]).max()
    assert np.all(pv >= 0) and pv.max() > 0
    s.close()


def test_snapshot_equals_the_strided_field():
    m, s = _run()
    start, count, stride = (3, 4, 5), (10, 7, 4), (2, 3, 4)
    snap = s.snapshot(start, count, stride, comps=(0, 4, 8))
    for q, c in enumerate((0, 4, 8)):
        f = s.get_field(c)
        ref = f[start[0]:start[0] + count[0] * stride[0]:stride[0],
                start[1]:start[1] + count[1] * stride[1]:stride[1],
                start[2]:start[2] + count[2] * stride[2]:stride[2]]
        assert np.array_equal(snap[q], ref)
    with pytest.raises(cgfd.CgfdError):
        s.snapshot((0, 0, 0), (1000, 1, 1))
    s.close()


def test_seismo_and_peakvel_netcdf_files(tmp_path):
    from scipy.io import netcdf_file
    m, s = _run(steps=25, pgv=True)
    pos = np.arange(3 * len(m.rcv_loc), dtype=np.float32) * 10.0
    p1, p2 = str(tmp_path / "seismo.nc"), str(tmp_path / "peakvel.nc")
    s.write_seismograms_nc(p1, pos)
    s.write_peak_velocity_nc(p2)
    seis = s.seismograms()
    with netcdf_file(p1, "r", mmap=False) as f:
        assert f.dimensions["PointNum"] == len(m.rcv_loc)
        assert f.variables["Vx"].shape == (25, len(m.rcv_loc))
        for c, name in enumerate(cgfd.COMPONENTS):
            assert np.array_equal(f.variables[name][:], seis[c, :, :25].T)
        t = f.variables["currTime"][:]
        assert np.allclose(t, (np.arange(25) + 1) * m.stept, rtol=1e-6)
        assert list(f.variables["Pnum"][:]) == list(range(1, len(m.rcv_loc) + 1))
        assert np.array_equal(f.variables["posy"][:], pos.reshape(-1, 3)[:, 1])
        assert f.Content.startswith(b"Velocity and Stress seismogram")
    pv = s.peak_velocity()
    with netcdf_file(p2, "r", mmap=False) as f:
        for c, name in enumerate(("Vx", "Vy", "Vz")):
            assert np.array_equal(f.variables[name][:], pv[c])
    s.close()
