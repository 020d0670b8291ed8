"""The host program (copara-cgfd3d_b200/wavesim_b200) in the tests: run it
on a par-file set and read its --dump output back as a models.Model."""
import os
import shutil
import subprocess

import numpy as np

import models

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "copara-cgfd3d_b200", "wavesim_b200")
PARFILES = os.path.join(ROOT, "tests", "golden", "parfiles")


def copy_parfiles(dst):
    """The par-file set copied into dst (the host writes its outputs next
    to the par files unless told otherwise)."""
    shutil.copytree(PARFILES, dst, dirs_exist_ok=True)
    return dst


def run(conf_dir, *args, timeout=600):
    p = subprocess.run([HOST, "SeisFD3D.conf", *args], cwd=conf_dir, capture_output=True,
                       text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(f"wavesim_b200 failed ({p.returncode}): {p.stdout}\n{p.stderr}")
    return p.stdout


def read_dump(path):
    """The pre-processed model of `wavesim_b200 --dump` as a dict."""
    with open(path, "rb") as f:
        hdr = np.frombuffer(f.read(48), np.int32)
        dd = np.frombuffer(f.read(24), np.float64)

        def vec(dtype):
            n = int(np.frombuffer(f.read(8), np.int64)[0])
            return np.frombuffer(f.read(n * np.dtype(dtype).itemsize), dtype).copy()

        ni, nj, nk, nt, con = (int(v) for v in hdr[:5])
        shape = (ni + 6, nj + 6, nk + 6)
        d = dict(ni=ni, nj=nj, nk=nk, nt=nt, con=con, nabs=tuple(int(v) for v in hdr[5:11]),
                 nfoc=int(hdr[11]), steph=float(dd[0]), stept=float(dd[1]), fdt=float(dd[2]))
        for k in ("x", "y", "z", "zeta_x", "zeta_y", "zeta_z", "jac"):
            d[k] = vec(np.float64).reshape(shape)
        for k in ("alpha", "beta", "rho"):
            d[k] = vec(np.float32).reshape(shape)
        d["pml"] = [vec(np.float64) for _ in range(9)]
        d["mloc"] = vec(np.int32).reshape(-1, 3)
        d["m6"] = vec(np.float32).reshape(-1, 6)
        d["mstf"] = vec(np.float32).reshape(len(d["mloc"]), -1)
        d["floc"] = vec(np.int32).reshape(-1, 3)
        d["f3"] = vec(np.float32).reshape(-1, 3)
        d["fstf"] = vec(np.float32).reshape(len(d["floc"]), -1)
        d["focloc"] = vec(np.int32).reshape(-1, 3)
        d["focmom"] = vec(np.float32)
        d["rloc"] = vec(np.int32).reshape(-1, 3)
        d["rpos"] = vec(np.float32).reshape(-1, 3)
    return d


def to_model(d, name="parfiles"):
    """The dumped arrays as a models.Model (the same inputs the host uploads)."""
    nstf = 2 * (d["nt"] + 1)
    empty = np.zeros((0, 3), np.int32)
    p = d["pml"]
    m = models.Model(
        name, d["ni"], d["nj"], d["nk"], d["steph"], d["stept"], d["nt"], d["con"], d["nabs"],
        dict(zeta_x=d["zeta_x"], zeta_y=d["zeta_y"], zeta_z=d["zeta_z"], jac=d["jac"]),
        d["alpha"], d["beta"], d["rho"], ((p[0], p[1], p[2]), (p[3], p[4], p[5]),
                                          (p[6], p[7], p[8])),
        d["mloc"] if len(d["mloc"]) else empty, d["m6"],
        d["mstf"] if len(d["mloc"]) else np.zeros((0, nstf), np.float32),
        d["floc"] if len(d["floc"]) else empty, d["f3"],
        d["fstf"] if len(d["floc"]) else np.zeros((0, nstf), np.float32), d["rloc"])
    return m
