"""The host program wavesim_b200 end to end on the GPU: the par-file set of
tests/golden/parfiles run through the C ABI, its seismo.nc, peakvel.nc and
snap_NNN.nc outputs read back with scipy and compared with the reference's
own runtime (oracle/_ref/ref_wavesim) run on the model the host built (its
--dump), within the 1e-5 parity bar: seismograms of the receivers and the
receiver line, the peak velocities, and the snapshot of an x-plane every 20
steps (SWpick)."""
import os

import numpy as np
import pytest

import cgfd
import hostio
import refio
from helpers import comp_errors, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


def test_host_outputs_match_the_reference_runtime(tmp_path):
    from scipy.io import netcdf_file
    d = hostio.copy_parfiles(str(tmp_path / "par"))
    hostio.run(d, "--dump", "model.bin")
    dump = hostio.read_dump(os.path.join(d, "model.bin"))
    m = hostio.to_model(dump)
    out = str(tmp_path / "out")
    os.makedirs(out)
    log = hostio.run(d, "--out", out)
    assert "0 non-finite" in log

    import make_parfiles as mp
    s2 = mp.SNAPS[1]
    start = [s2[a] - 1 + 3 for a in range(3)]
    count, stride, tinv = s2[3:6], s2[6:9], s2[9]
    ax = [start[a] + stride[a] * np.arange(count[a]) for a in range(3)]
    g = np.meshgrid(*ax, indexing="ij")
    pts = np.stack([a.reshape(-1) for a in g], axis=1).astype(np.int32)
    r = refio.run(m, m.nt, fields=False, peak_velocity=True, snap_points=pts, snap_tinv=tinv)

    with netcdf_file(os.path.join(out, "seismo.nc"), "r", mmap=False) as f:
        seis = np.stack([np.array(f.variables[n][:]).T for n in cgfd.COMPONENTS])
        assert list(f.variables["Lnum"][:]) == [0] * len(mp.RECV) + [1] * mp.LINES[0][2]
        assert np.allclose(f.variables["posz"][:], dump["rpos"][:, 2])
    assert seis.shape == r["seis"].shape and np.abs(r["seis"][:3]).max() > 0
    for c in range(3):
        assert rel_l2(seis[c], r["seis"][c]) < TOL, cgfd.COMPONENTS[c]
    for c, e in enumerate(comp_errors(seis, r["seis"])):
        assert e < TOL, (cgfd.COMPONENTS[c], e)

    with netcdf_file(os.path.join(out, "peakvel.nc"), "r", mmap=False) as f:
        pv = np.stack([np.array(f.variables[n][:]) for n in ("Vx", "Vy", "Vz")])
    ref_pv = r["pv"][:, 3:-3, 3:-3]
    for c in range(3):
        assert rel_l2(pv[c], ref_pv[c]) < TOL, c

    with netcdf_file(os.path.join(out, "snap_002.nc"), "r", mmap=False) as f:
        snap = np.stack([np.array(f.variables[n][:]).reshape(-1, len(pts)).T
                         for n in cgfd.COMPONENTS])
        assert len(f.variables["time"][:]) == r["snap"].shape[2]
    for c, e in enumerate(comp_errors(snap, r["snap"])):
        assert e < TOL, (cgfd.COMPONENTS[c], e)
    with netcdf_file(os.path.join(out, "snap_001.nc"), "r", mmap=False) as f:
        assert set(f.variables) >= {"Vx", "Vy", "Vz"} and "Txx" not in f.variables
        assert f.variables["Vz"].shape == (10, mp.NI, mp.NJ, 1)
