"""Generates the vmap-grid fixtures (tests/golden/grid_vmap_*.npz): vmap
descriptions run through the reference's own gridmesh (oracle/_ref/ref_grid,
built by oracle/ref/Makefile from the reference's sources in its
double-precision configuration), inputs and outputs saved together: the
node coordinates and ConIndex (read_vmapnew), the metric of that grid
(calmetric: xi, eta, zeta derivatives and the Jacobian, steph 100) and its
ADE CFS-PML profiles (absorb::CalCFSfactors: APD, B, DB per axis).

Run from the repository root after `make -C oracle/ref`:
    python tests/golden/make_grid_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.path.join(ROOT, "oracle", "_ref", "ref_grid")
OUT = os.path.dirname(os.path.abspath(__file__))


def anchors(ni, nj, tops, seed):
    """Interface depths per column: a smooth random perturbation around each
    mean depth, the surface with a hill."""
    rng = np.random.default_rng(seed)
    h = 100.0
    a = np.zeros((ni, nj, 2 + len(tops)))
    ii, jj = np.meshgrid(np.arange(ni), np.arange(nj), indexing="ij")
    a[..., 0] = ii * h
    a[..., 1] = jj * h
    for q, zm in enumerate(tops):
        amp = 300.0 if q == 0 else 80.0
        ph = rng.uniform(0, 2 * np.pi, 2)
        a[..., 2 + q] = zm + amp * np.sin(ii / ni * 3.0 + ph[0]) * np.cos(jj / nj * 2.0 + ph[1])
    return a


CASES = {
    # a graded layer between equally spaced ones (geometric branch)
    "grid_vmap_graded": dict(ni=9, nj=7, gp=[6, 10, 8], eq=[1, 0, 1],
                             tops=[0.0, -900.0, -3000.0, -6000.0], hybrid=0, depth=0.0, seed=1),
    # a graded layer whose mean spacing lies outside its neighbours' (ramp branch)
    "grid_vmap_ramp": dict(ni=8, nj=6, gp=[4, 16, 4], eq=[1, 0, 1],
                           tops=[0.0, -1200.0, -2000.0, -3600.0], hybrid=0, depth=0.0, seed=2),
    # hybrid: flat below the conversion depth, layers re-cut in proportion
    "grid_vmap_hybrid": dict(ni=9, nj=7, gp=[6, 10, 8], eq=[1, 1, 1],
                             tops=[0.0, -900.0, -3000.0, -6000.0], hybrid=1, depth=-2000.0,
                             seed=3),
    # hybrid with a graded layer above the conversion interface
    "grid_vmap_hybrid_graded": dict(ni=8, nj=8, gp=[5, 8, 6, 6], eq=[1, 0, 1, 1],
                                    tops=[0.0, -700.0, -2200.0, -3500.0, -5000.0], hybrid=1,
                                    depth=-2800.0, seed=4),
}


# CFS-PML parameters for absorb::CalCFSfactors on each grid (small layers:
# the grids are 6-9 nodes wide)
PML = dict(nabs=(3, 2, 2, 2, 4, 0), velabs=6000.0, bmax=2.5, amax=5.0, stept=0.008)


def run_reference(ni, nj, nk, gp, eq, a, hybrid, depth):
    with tempfile.TemporaryDirectory(prefix="g", dir="/tmp") as d:
        with open(os.path.join(d, "grid.dat"), "w") as f:
            f.write("#grid vmap\n")
            f.write(f"vmap_dims = {ni} {nj} {a.shape[-1] - 2}\n")
            f.write("vmap_gridpoints = " + " ".join(map(str, gp)) + "\n")
            f.write("vmap_equalspacing = " + " ".join(map(str, eq)) + "\n")
            f.write("<vmap_anchor>\n")
            for i in range(ni):
                for j in range(nj):
                    f.write(" ".join(f"{v:.17g}" for v in a[i, j]) + "\n")
        out, met, pml = (os.path.join(d, f) for f in ("out.bin", "met.bin", "pml.bin"))
        subprocess.run([REF, d, str(ni), str(nj), str(nk), str(hybrid), repr(float(depth)), out,
                        met, pml, *map(str, PML["nabs"]), repr(PML["velabs"]),
                        repr(PML["bmax"]), repr(PML["amax"]), repr(PML["stept"])],
                       check=True, stdout=subprocess.DEVNULL)
        raw = open(out, "rb").read()
        metric = np.fromfile(met, np.float64).reshape(10, ni + 6, nj + 6, nk + 6)
        p = np.fromfile(pml, np.float64)
        n3 = (ni + 6, nj + 6, nk + 6)
        cfs, o = [], 0
        for ax in range(3):
            cfs.append(p[o:o + 3 * n3[ax]].reshape(3, n3[ax]))  # APD, B, DB
            o += 3 * n3[ax]
    con = int(np.frombuffer(raw[:4], np.int32)[0])
    xyz = np.frombuffer(raw[4:], np.float64).reshape(3, ni + 6, nj + 6, nk + 6)
    return con, xyz, metric, cfs


def main():
    for name, c in CASES.items():
        a = anchors(c["ni"], c["nj"], c["tops"], c["seed"])
        nk = sum(c["gp"]) + 1
        con, xyz, metric, cfs = run_reference(c["ni"], c["nj"], nk, c["gp"], c["eq"], a,
                                              c["hybrid"], c["depth"])
        np.savez_compressed(os.path.join(OUT, name + ".npz"), ni=c["ni"], nj=c["nj"], nk=nk,
                            gridpoints=np.array(c["gp"], np.int32),
                            equalspacing=np.array(c["eq"], np.int32), anchor=a,
                            hybrid=c["hybrid"], depth=c["depth"], con_index=con, x=xyz[0],
                            y=xyz[1], z=xyz[2], metric=metric, pml_nabs=np.array(PML["nabs"]),
                            pml_velabs=PML["velabs"], pml_bmax=PML["bmax"],
                            pml_amax=PML["amax"], pml_x=cfs[0], pml_y=cfs[1], pml_z=cfs[2])
        print(name, "ConIndex", con)


if __name__ == "__main__":
    sys.exit(main())
