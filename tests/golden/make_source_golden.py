"""Generates the source fixtures: node coordinates, source and receiver
positions run through the reference's own source location and smoothing
(tests/golden/source_locate_*.npz), and its source time functions of every
wavelet type and strike/dip/rake moment tensors (tests/golden/
source_wavelets.npz), by oracle/_ref/ref_source, built by
oracle/ref/Makefile from the reference's source.cpp, common.cpp and
mathfunc.cpp with its SrcSmooth and TypeDouble options; inputs and outputs
saved together.

Run from the repository root after `make -C oracle/ref`:
    python tests/golden/make_source_golden.py
"""
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.path.join(ROOT, "oracle", "_ref", "ref_source")
OUT = os.path.dirname(os.path.abspath(__file__))


def hill_grid(ni, nj, nk, h, wobble, seed):
    """Full node arrays (ni+6, nj+6, nk+6), z fastest: a Gaussian hill on top,
    vertical spacing stretched with depth, x and y on steph (wobble = 0) or
    displaced by up to wobble*h (a general curvilinear grid)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = ni + 6, nj + 6, nk + 6
    i = (np.arange(nx) - 3.0)[:, None, None]
    j = (np.arange(ny) - 3.0)[None, :, None]
    k = (np.arange(nz) - 3.0)[None, None, :]
    cx, cy = (ni - 1) * h / 2, (nj - 1) * h / 2
    x = np.broadcast_to(i * h, (nx, ny, nz)).copy()
    y = np.broadcast_to(j * h, (nx, ny, nz)).copy()
    if wobble:
        ph = rng.uniform(0, 2 * np.pi, 4)
        x += wobble * h * np.sin(0.7 * j + ph[0]) * np.cos(0.5 * k + ph[1])
        y += wobble * h * np.cos(0.6 * i + ph[2]) * np.sin(0.4 * k + ph[3])
    top = 0.8 * h * nk * 0.25 * np.exp(-((i * h - cx) ** 2 + (j * h - cy) ** 2) / (0.3 * ni * h) ** 2)
    depth = h * nk
    s = (nk - 1 - k) / (nk - 1)  # 0 at the surface, 1 at the bottom
    z = top - depth * (0.6 * s + 0.4 * s * s) * (1.0 + 0.2 * top / depth)
    return x, y, np.broadcast_to(z, (nx, ny, nz)).copy()


CASES = {
    # flat-spaced x, y (the solver's SimpleCar grids) with a hill on top
    "source_locate_hill": dict(ni=14, nj=12, nk=12, h=100.0, wobble=0.0, seed=11, nf=5, nm=5,
                               nr=12),
    # x, y displaced along the other axes: a general curvilinear grid
    "source_locate_curved": dict(ni=12, nj=13, nk=12, h=80.0, wobble=0.15, seed=12, nf=5, nm=5,
                                 nr=12),
}


def points(x, y, z, n, rng, margin, hyp=None, frac_above=0.0):
    """n positions inside the valid nodes (margin nodes from the x-y sides
    and the bottom), some of them just below the surface; with hyp, a
    fraction is put above hyper_height."""
    ni, nj, nk = (d - 6 for d in x.shape)
    out = []
    for q in range(n):
        i = rng.uniform(3 + margin, ni + 2 - margin)
        j = rng.uniform(3 + margin, nj + 2 - margin)
        if q % 3 == 0:
            k = nk + 2 - rng.uniform(0.6, 2.4)  # block reaches above the surface
        else:
            k = rng.uniform(3 + 4, nk + 2 - 3)
        ii, jj, kk = int(round(i)), int(round(j)), int(round(k))
        p = [np.interp(i, [ii - 1, ii, ii + 1], x[ii - 1:ii + 2, jj, kk]),
             np.interp(j, [jj - 1, jj, jj + 1], y[ii, jj - 1:jj + 2, kk]),
             np.interp(k, [kk - 1, kk, kk + 1], z[ii, jj, kk - 1:kk + 2])]
        if hyp is not None and rng.uniform() < frac_above:
            p[2] = hyp + rng.uniform(10.0, 500.0)
        out.append(p)
    return np.array(out, np.float64)


def run_reference(x, y, z, rho, vs, hyp, stept, nt, forces, moments, recv, opts=()):
    ni, nj, nk = (d - 6 for d in x.shape)
    with tempfile.TemporaryDirectory(prefix="s", dir="/tmp") as d:
        inp = os.path.join(d, "in.bin")
        with open(inp, "wb") as f:
            np.array([ni, nj, nk, len(forces), len(moments), len(recv), nt], np.int32).tofile(f)
            np.array([hyp, stept], np.float64).tofile(f)
            for a in (x, y, z, rho, vs):
                np.ascontiguousarray(a, np.float64).tofile(f)
            for a in (forces, moments, recv):
                np.ascontiguousarray(a, np.float64).tofile(f)
        out = os.path.join(d, "out.bin")
        subprocess.run([REF, d, inp, out, *map(str, opts)], check=True, stdout=subprocess.DEVNULL)
        raw = open(out, "rb").read()
    nstf = 2 * (nt + 1)
    rec_frc = np.dtype([("loc", "<i4", 3), ("posz", "<f8"), ("dnorm", "<f8", 343),
                        ("stf", "<f8", nstf), ("coef", "<f8", 3)])
    rec_mnt = np.dtype([("loc", "<i4", 3), ("posz", "<f8"), ("dnorm", "<f8", 343),
                        ("stf", "<f8", nstf), ("coef", "<f8", 6)])
    rec_pt = np.dtype([("loc", "<i4", 3), ("posz", "<f8")])
    o = 0
    fr = np.frombuffer(raw, rec_frc, len(forces), o)
    o += fr.nbytes
    mr = np.frombuffer(raw, rec_mnt, len(moments), o)
    o += mr.nbytes
    rr = np.frombuffer(raw, rec_pt, len(recv), o)
    assert o + rr.nbytes == len(raw)
    return fr, mr, rr


def main():
    for name, c in CASES.items():
        rng = np.random.default_rng(c["seed"])
        x, y, z = hill_grid(c["ni"], c["nj"], c["nk"], c["h"], c["wobble"], c["seed"])
        rho = np.full(x.shape, 2600.0)
        vs = np.full(x.shape, 3000.0)
        hyp = float(z[3:-3, 3:-3, -4].max()) + 50.0
        nt, stept = 40, 0.008
        fpos = points(x, y, z, c["nf"], rng, 1)
        mpos = points(x, y, z, c["nm"], rng, 1)
        rpos = points(x, y, z, c["nr"], rng, 0, hyp, 0.5)
        forces = np.concatenate([fpos, rng.normal(size=(len(fpos), 3))], axis=1)
        moments = np.concatenate([mpos, rng.normal(size=(len(mpos), 6))], axis=1)
        fr, mr, rr = run_reference(x, y, z, rho, vs, hyp, stept, nt, forces, moments, rpos)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), x=x, y=y, z=z, hyp=hyp,
                            stept=stept, nt=nt, force_pos=fpos, moment_pos=mpos, recv_pos=rpos,
                            force_loc=fr["loc"], force_posz=fr["posz"],
                            force_w=fr["dnorm"].reshape(-1, 7, 7, 7), force_stf=fr["stf"],
                            moment_loc=mr["loc"], moment_posz=mr["posz"],
                            moment_w=mr["dnorm"].reshape(-1, 7, 7, 7), moment_stf=mr["stf"],
                            recv_loc=rr["loc"], recv_posz=rr["posz"])
        print(name, "done")
    wavelets()


# wavelet types with (time factor t0, frequency factor f0) for each; start
# times 0 and 0.05 s
WAVELETS = {"Gauss": (0.3, 0.08), "gauss": (0.3, 0.08), "Ricker": (0.6, 2.0),
            "ricker": (0.6, 2.0), "Bell": (0.1, 0.4), "bell": (0.1, 0.4), "BELL": (0.1, 0.4),
            "Step": (0.0, 1.0)}
ANGLES = [(30.0, 60.0, 90.0), (0.0, 90.0, 0.0), (123.0, 35.0, -71.0), (270.0, 10.0, 180.0)]


def wavelets():
    """One force and the ANGLES moments (moment_mech_input = angle) on a
    small flat grid, once per wavelet type and start time: the reference's
    sampled force and moment STFs and its moment tensors (x mu)."""
    x, y, z = hill_grid(8, 8, 8, 100.0, 0.0, 1)
    z = z - z[3:-3, 3:-3, -4].max()  # highest surface node at z = 0
    rho = np.full(x.shape, 2500.0)
    vs = np.full(x.shape, 3000.0)
    nt, stept = 80, 0.01
    c = [float(x[6, 6, 6]), float(y[6, 6, 6]), float(z[6, 6, 6])]
    forces = np.array([c + [1.0, -2.0, 0.5]])
    moments = np.array([c + list(a) + [0.0, 0.0, 0.0] for a in ANGLES])
    out = dict(nt=nt, stept=stept, angles=np.array(ANGLES), mu=2500.0 * 3000.0 ** 2)
    for start in (0.0, 0.05):
        for name, (t0, f0) in WAVELETS.items():
            fr, mr, _ = run_reference(x, y, z, rho, vs, 1e9, stept, nt, forces, moments,
                                      np.zeros((0, 3)),
                                      (name, t0, f0, name, t0, f0, "angle", start))
            key = f"{name}_{start:g}"
            out["force_" + key] = fr["stf"][0]
            out["moment_" + key] = mr["stf"][0]
            out["t0f0_" + name] = np.array([t0, f0])
            out["m6"] = mr["coef"]
    np.savez_compressed(os.path.join(OUT, "source_wavelets.npz"), **out)
    print("source_wavelets done")


if __name__ == "__main__":
    main()
