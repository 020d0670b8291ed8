"""The NetCDF classic readers of the reference's model inputs
(cgfd_read_media_volume_nc, cgfd_read_focal_nc) against files written by
scipy's independent NetCDF writer: both classic versions, a record
dimension, the value types the format has, and the errors (missing
variables, NetCDF-4/HDF5 files, wrong shapes)."""
import os

import numpy as np
import pytest

import cgfd


def _write_volume(path, version=2, dtype="f4", zname="depth", shape=(5, 4, 6), seed=0):
    from scipy.io import netcdf_file
    rng = np.random.default_rng(seed)
    ax = [np.sort(rng.uniform(-1e3, 1e3, n)) for n in shape]
    vol = {k: rng.uniform(1.0, 8.0, shape).astype(np.float32) for k in ("Vp", "Vs", "rho")}
    with netcdf_file(path, "w", version=version) as f:
        for name, a in zip(("x", "y", zname), ax):
            f.createDimension(name, len(a))
            v = f.createVariable(name, "f8", (name,))
            v[:] = a
        for k, a in vol.items():
            v = f.createVariable(k, dtype, ("x", "y", zname))
            v[:] = a.astype(dtype)
    return ax, vol


@pytest.mark.parametrize("version", [1, 2])
@pytest.mark.parametrize("dtype", ["f4", "f8", "i2", "i4"])
def test_volume_media_round_trip(tmp_path, version, dtype):
    p = str(tmp_path / "v.nc")
    ax, vol = _write_volume(p, version, dtype)
    vx, vy, vz, vp, vs, rho = cgfd.read_media_volume_nc(p)
    for a, b in zip((vx, vy, vz), ax):
        assert np.array_equal(a, b)
    for a, k in zip((vp, vs, rho), ("Vp", "Vs", "rho")):
        assert np.array_equal(a, vol[k].astype(dtype).astype(np.float32))


def test_volume_media_z_axis_name(tmp_path):
    p = str(tmp_path / "v.nc")
    ax, vol = _write_volume(p, zname="z")
    vz = cgfd.read_media_volume_nc(p)[2]
    assert np.array_equal(vz, ax[2])


def _write_focal(path, npt=3, nt=9, record=False, dt=0.006, seed=1):
    from scipy.io import netcdf_file
    rng = np.random.default_rng(seed)
    mom = rng.standard_normal((6, npt, nt)).astype(np.float32) * 1e15
    pos = rng.uniform(-5e3, 5e3, (npt, 3))
    names = ("Mxx", "Myy", "Mzz", "Mxy", "Mxz", "Myz")
    with netcdf_file(path, "w", version=2) as f:
        f.createDimension("NP", None if record else npt)
        f.createDimension("NT", nt)
        f.DT = np.float64(dt)
        for c, n in enumerate(names):
            v = f.createVariable(n, "f4", ("NP", "NT"))
            v[:] = mom[c]
        for a, n in enumerate(("posx", "posy", "posz")):
            v = f.createVariable(n, "f8", ("NP",))
            v[:] = pos[:, a]
    return mom, pos


@pytest.mark.parametrize("record", [False, True])
def test_focal_series_round_trip(tmp_path, record):
    p = str(tmp_path / "f.nc")
    mom, pos = _write_focal(p, record=record)
    dt, got_pos, got = cgfd.read_focal_nc(p)
    assert dt == 0.006
    assert np.array_equal(got, mom) and np.array_equal(got_pos, pos)


def test_reader_errors(tmp_path):
    hdf = str(tmp_path / "h.nc")
    with open(hdf, "wb") as f:
        f.write(b"\x89HDF\r\n\x1a\n" + bytes(64))
    with pytest.raises(cgfd.CgfdError, match="nccopy -k classic"):
        cgfd.read_media_volume_nc(hdf)
    p = str(tmp_path / "v.nc")
    _write_volume(p)
    with pytest.raises(cgfd.CgfdError, match="NP and NT"):
        cgfd.read_focal_nc(p)
    q = str(tmp_path / "nodt.nc")
    from scipy.io import netcdf_file
    with netcdf_file(q, "w") as f:
        f.createDimension("NP", 2)
        f.createDimension("NT", 3)
    with pytest.raises(cgfd.CgfdError, match="DT"):
        cgfd.read_focal_nc(q)
    with pytest.raises(cgfd.CgfdError, match="cannot open"):
        cgfd.read_focal_nc(str(tmp_path / "missing.nc"))


def test_readers_refuse_mismatched_sizes(tmp_path):
    import ctypes as C
    p = str(tmp_path / "v.nc")
    _write_volume(p, shape=(3, 3, 3))
    n = [C.c_int(4), C.c_int(3), C.c_int(3)]
    buf = np.zeros(64)
    f = np.zeros(64, np.float32)
    st = cgfd._lib.cgfd_read_media_volume_nc(p.encode(), *[C.byref(x) for x in n],
                                             *[cgfd._d(buf)] * 3, *[cgfd._f(f)] * 3)
    assert st == cgfd.ERR_ARG and "sizes differ" in cgfd.last_error(None)
    assert os.path.exists(p)


def _damage_dims(raw, lens):
    """raw with the lengths of the CDF-2 header's dimensions x and y replaced
    (a dimension entry: name length, name padded to 4 bytes, length)."""
    for (name, n), new in zip(((b"x", 5), (b"y", 4)), lens):
        entry = (1).to_bytes(4, "big") + name + b"\0\0\0" + n.to_bytes(4, "big")
        assert raw.count(entry) == 1
        raw = raw.replace(entry, entry[:-4] + new.to_bytes(4, "big"))
    return raw


def test_readers_refuse_data_outside_the_file(tmp_path):
    """A truncated file, and damaged headers whose dimensions claim more data
    than the file holds, are refused before anything is allocated or
    written: 2^31-1 x 2^31-1 x 6 values (a count that overflows 64 bits) at
    the size query, 2^24 x 4 x 6 values when the variables are read."""
    import ctypes as C
    p = str(tmp_path / "v.nc")
    _write_volume(p)
    raw = open(p, "rb").read()
    t = str(tmp_path / "truncated.nc")
    with open(t, "wb") as f:
        f.write(raw[:-100])
    with pytest.raises(cgfd.CgfdError, match="outside the file"):
        cgfd.read_media_volume_nc(t)
    d = str(tmp_path / "overflow.nc")
    with open(d, "wb") as f:
        f.write(_damage_dims(raw, (0x7FFFFFFF, 0x7FFFFFFF)))
    with pytest.raises(cgfd.CgfdError, match="overflows"):
        cgfd.read_media_volume_nc(d)
    d = str(tmp_path / "damaged.nc")
    with open(d, "wb") as f:
        f.write(_damage_dims(raw, (1 << 24, 4)))
    n = [C.c_int(0) for _ in range(3)]
    st = cgfd._lib.cgfd_read_media_volume_nc(d.encode(), *[C.byref(x) for x in n], None, None,
                                             None, None, None, None)
    assert st == 0 and [x.value for x in n] == [1 << 24, 4, 6]
    small = [np.zeros(8) for _ in range(3)] + [np.zeros(8, np.float32) for _ in range(3)]
    ptrs = [cgfd._d(a) for a in small[:3]] + [cgfd._f(a) for a in small[3:]]
    st = cgfd._lib.cgfd_read_media_volume_nc(d.encode(), *[C.byref(x) for x in n], *ptrs)
    assert st == cgfd.ERR_ARG
    assert "outside the file" in cgfd.last_error(None)
    assert all(not a.any() for a in small)
