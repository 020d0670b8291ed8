"""Writes the small par-file set of the host program's tests
(tests/golden/parfiles/): the reference's SeisFD3D.conf, a vmap grid file
with a Gaussian hill (hybrid grid), a volume media file in NetCDF classic
format, absorb.dat, source.dat (one force, two moments given by strike / dip
/ rake) and station.dat (receivers, a receiver line, two snapshots), in the
formats the reference reads (src/simulation.cc:759-790, gridmesh.cpp:84-130,
mediaparas.cpp:1273-1425, absorb.cpp:26-44, source.cpp:686-790,
seisplot.cpp:336-420).  Then runs the reference's own vmap reader, grid
generation, calmetric and CalCFSfactors (oracle/_ref/ref_grid, built by
oracle/ref/Makefile from its sources) on the same vmap file and absorb
parameters and saves the result as tests/golden/parfiles_ref_grid.npz.

Run from the repository root after `make -C oracle/ref`:
    python tests/golden/make_parfiles.py
"""
import os
import shutil
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "parfiles")
REF_GRID = os.path.join(ROOT, "oracle", "_ref", "ref_grid")

NI, NJ, NK, NT = 48, 40, 32, 100
STEPH, STEPT = 100.0, 0.008
CONVERS = -1500.0
NABS = (6, 6, 6, 6, 6, 0)
VEL, BMAX, AMAX = 5000.0, 2.5, 5.0


def hill(x, y):
    return 350.0 * np.exp(-((x - 300.0) ** 2 + (y + 200.0) ** 2) / 1200.0 ** 2)


def write_conf(d):
    with open(os.path.join(d, "SeisFD3D.conf"), "w") as f:
        f.write(f"""#######################################################################
#  small hill model for the host program's tests (tests/golden/make_parfiles.py)
#######################################################################
BlockPerGrid = 64 32 1
ThreadPerBlock = 256 1 1
ni    = {NI}
nj    = {NJ}
nk    = {NK}
nt    = {NT}
stept = {STEPT}
steph = {STEPH}
seispath = .
device_filename = device.dat
grid_type = vmap  # vmap or point
grid_filename = grid_vmap.dat
hybrid_grid = 1
conversion_interface_depth = {CONVERS:.1f}
reference_velocity = 2000.0
media_type = volume # interface, interface3D or volume
media_filename = media_volume.nc
threshold_velocity_jump_of_interface = 100
threshold_percent_change_of_interface = 0.1
sampling_point_per_cell = 0 0 0
source_filename = source.dat
station_filename = station.dat
output_peakvel = 1 # 1 YES 0 NO
full_wave_field_storage_interval = 1000000
absorb_filename = absorb.dat
""")


def write_grid(d):
    x = -2350.0 + STEPH * np.arange(NI)
    y = -1950.0 + STEPH * np.arange(NJ)
    with open(os.path.join(d, "grid_vmap.dat"), "w") as f:
        f.write("#grid vmap ascii data\n")
        f.write(f"vmap_dims = {NI} {NJ} 2\nvmap_gridpoints = {NK - 1}\nvmap_equalspacing = 1\n")
        f.write("#from top to bottom, Xcord Ycord Zsurf1 Zsurf2\n<vmap_anchor>\n")
        for i in range(NI):
            for j in range(NJ):
                f.write(f"{x[i]:.6f} {y[j]:.6f} {hill(x[i], y[j]):.6f} -3100.000000\n")


def write_media(d):
    from scipy.io import netcdf_file
    vx = np.arange(-3000.0, 3000.1, 500.0)
    vy = np.arange(-2500.0, 2500.1, 500.0)
    vz = np.arange(-3500.0, 1000.1, 250.0)
    z = vz[None, None, :]
    xx = vx[:, None, None]
    vp = np.where(z > -1200.0, 3500.0 + 0.1 * xx, 5000.0 - 0.3 * (z + 1200.0))
    vp = np.broadcast_to(vp, (len(vx), len(vy), len(vz))).astype(np.float32)
    vs = (vp / 1.73).astype(np.float32)
    rho = (2300.0 + 0.1 * vp).astype(np.float32)
    with netcdf_file(os.path.join(d, "media_volume.nc"), "w", version=2) as f:
        for name, ax in (("x", vx), ("y", vy), ("depth", vz)):
            f.createDimension(name, len(ax))
            v = f.createVariable(name, "f4", (name,))
            v[:] = ax
        for name, a in (("Vp", vp), ("Vs", vs), ("rho", rho)):
            v = f.createVariable(name, "f4", ("x", "y", "depth"))
            v[:] = a


def write_absorb(d):
    with open(os.path.join(d, "absorb.dat"), "w") as f:
        f.write("#X1 X2 Y1 Y2 Z1 Z2(from index smal to large)\n")
        f.write("abs_number = " + " ".join(str(n) for n in NABS) + "\n")
        f.write("abs_velocity  = " + " ".join([f"{VEL:.0f}"] * 6) + "\n")
        f.write("bmax = " + " ".join([str(BMAX)] * 6) + "\n")
        f.write("amax = " + " ".join([str(AMAX)] * 6) + "\n")


# force: x y z (km) | start | f0 | fx fy fz ; moments (angle): x y z | start | m0 | s d r
FORCES = [(0.4, -0.3, -1.2, 0.0, 1.0e15, 0.3, -0.2, 1.0)]
MOMENTS = [(-0.5, 0.4, -1.8, 0.02, 1.0e15, 30.0, 60.0, 90.0),
           (0.9, 0.6, -2.2, 0.0, 2.0e15, 120.0, 45.0, -30.0)]
FORCE_STF = ("Gauss", 0.25, 0.06)
MOMENT_STF = ("Ricker", 0.3, 4.0)


def write_source(d):
    with open(os.path.join(d, "source.dat"), "w") as f:
        f.write("source_hyper_height = 9.0\ndistance2meter = 1.0E3\n")
        f.write("source_type = 3 # 1-> focal ; 2-> force ; 3-> moment\n")
        f.write("simulate_damp = 1.0\n")
        f.write(f"number_of_force_source = {len(FORCES)}\nforce_stf_window = 1\n")
        f.write(f"force_stf_type = {FORCE_STF[0]}\nforce_stf_timefactor = {FORCE_STF[1]}\n")
        f.write(f"force_stf_freqfactor = {FORCE_STF[2]}\n")
        f.write("# x,y,z           | start  | f0    | fx   fy   fz\n<anchor_force>\n")
        for r in FORCES:
            f.write("  " + "  ".join(f"{v:g}" for v in r) + "\n")
        f.write(f"number_of_moment_source = {len(MOMENTS)}\nmoment_stf_window = 1\n")
        f.write(f"moment_stf_type = {MOMENT_STF[0]}\nmoment_stf_timefactor = {MOMENT_STF[1]}\n")
        f.write(f"moment_stf_freqfactor = {MOMENT_STF[2]}\nmoment_mech_input = angle\n")
        f.write("# x,y,z     RuptT(s)    | m0(N.M) | strike dip rake\n<anchor_moment>\n")
        for r in MOMENTS:
            f.write("  " + "  ".join(f"{v:g}" for v in r) + "\n")


# snapshots: start (1-based valid index) | count | stride | tinv | cmp
SNAPS = [(1, 1, NK, NI, NJ, 1, 1, 1, 1, 10, 1),
         (24, 1, 1, 1, NJ // 2, NK // 2, 1, 2, 2, 20, 3)]
RECV = [(0.0, 0.0, 9000e3), (1.0e3, -0.5e3, 9000e3), (-0.5e3, 0.5e3, -1.0e3),
        (0.3e3, 0.3e3, -2.5e3)]
LINES = [((-1.5e3, 0.0, 9000e3), (0.5e3, 0.0, 0.0), 7)]


def write_station(d):
    with open(os.path.join(d, "station.dat"), "w") as f:
        f.write(f"number_of_snap = {len(SNAPS)}\n")
        f.write("# id        start          count           stride  tinv  cmp\n")
        for q, s in enumerate(SNAPS):
            f.write(f"snap_{q + 1:03d} = " + " ".join(str(v) for v in s) + "\n")
        f.write("topo_hyper_height = 8000.0E3\ntinv_of_seismo = 1\n")
        f.write(f"number_of_inline = {len(LINES)}\n")
        for q, (p0, dp, n) in enumerate(LINES):
            f.write(f"line_{q + 1:03d} = {p0[0]:g} {p0[1]:g} {p0[2]:g} | {dp[0]:g} {dp[1]:g} "
                    f"{dp[2]:g} | {n}\n")
        f.write(f"number_of_recv = {len(RECV)}\n")
        for q, r in enumerate(RECV):
            f.write(f"recv_{q + 1:03d} = {r[0]:g} {r[1]:g} {r[2]:g}\n")


def run_ref_grid(d):
    """The reference's reader, grid, metric and CFS-PML on grid_vmap.dat."""
    n = (NI + 6) * (NJ + 6) * (NK + 6)
    with tempfile.TemporaryDirectory(dir="/tmp") as td:
        shutil.copy(os.path.join(d, "grid_vmap.dat"), os.path.join(td, "grid.dat"))
        out, met, pml = (os.path.join(td, f) for f in ("g.bin", "m.bin", "p.bin"))
        subprocess.run([REF_GRID, td, str(NI), str(NJ), str(NK), "1", str(CONVERS), out, met, pml,
                        *[str(v) for v in NABS], str(VEL), str(BMAX), str(AMAX), str(STEPT)],
                       check=True, capture_output=True)
        raw = open(out, "rb").read()
        con = int(np.frombuffer(raw[:4], np.int32)[0])
        xyz = np.frombuffer(raw[4:], np.float64).reshape(3, NI + 6, NJ + 6, NK + 6)
        m = np.fromfile(met, np.float64).reshape(10, NI + 6, NJ + 6, NK + 6)
        p = np.fromfile(pml, np.float64)
    lens = [NI + 6, NJ + 6, NK + 6]
    pm, o = [], 0
    for q in range(9):
        ln = lens[q // 3]
        pm.append(p[o:o + ln])
        o += ln
    assert o == len(p) and n == xyz[0].size
    return dict(con=con, x=xyz[0], y=xyz[1], z=xyz[2], zeta_x=m[6], zeta_y=m[7], zeta_z=m[8],
                jac=m[9], apd_x=pm[0], b_x=pm[1], db_x=pm[2], apd_y=pm[3], b_y=pm[4],
                db_y=pm[5], apd_z=pm[6], b_z=pm[7], db_z=pm[8])


def main():
    os.makedirs(OUT, exist_ok=True)
    write_conf(OUT)
    write_grid(OUT)
    write_media(OUT)
    write_absorb(OUT)
    write_source(OUT)
    write_station(OUT)
    ref = run_ref_grid(OUT)
    np.savez_compressed(os.path.join(os.path.dirname(OUT), "parfiles_ref_grid.npz"), **ref)
    print("par files in", OUT, "ConIndex", ref["con"])


if __name__ == "__main__":
    main()
