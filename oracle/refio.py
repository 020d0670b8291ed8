"""Input/output of the reference parity driver (oracle/_ref/ref_wavesim).

TEST INFRASTRUCTURE ONLY.  write_input() serialises a model (the same arrays
that feed cgfd.Solver and the CPU oracle); run() executes the reference's own
ChildProcs time loop on the GPU (built by oracle/ref/Makefile from the
reference's sources); the result holds its seismograms (HPW layout) and the
final FW and W fields.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "ref_wavesim")
# the same runtime built with the reference's SrcSmooth option
REF_BIN_SMOOTH = os.path.join(HERE, "_ref", "ref_wavesim_smooth")
MAGIC = 0x52464743


def available() -> bool:
    return os.path.exists(REF_BIN)


def write_input(m, path, nsteps, init_fields=None, nstages=0):
    nstf = m.mnt_stf.shape[1] if len(m.mnt_loc) else (m.frc_stf.shape[1] if len(m.frc_loc) else 0)
    if len(m.mnt_loc) and len(m.frc_loc) and m.mnt_stf.shape[1] != m.frc_stf.shape[1]:
        raise ValueError("moment and force STFs must have the same length")
    hdr = [MAGIC, 1, m.ni, m.nj, m.nk, m.nt, nsteps, m.con_index, *m.nabs,
           len(m.mnt_loc), len(m.frc_loc), nstf, len(m.rcv_loc),
           1 if init_fields is not None else 0, nstages]
    f32 = lambda a: np.ascontiguousarray(a, np.float32).tobytes()
    i32 = lambda a: np.ascontiguousarray(a, np.int32).tobytes()
    with open(path, "wb") as f:
        f.write(struct.pack("<20i", *hdr))
        f.write(struct.pack("<2d", m.steph, m.stept))
        for k in ("zeta_x", "zeta_y", "zeta_z", "jac"):
            f.write(f32(m.metric[k]))
        for a in (m.alpha, m.beta, m.rho):
            f.write(f32(a))
        for group in m.pml:
            for a in group:
                f.write(f32(a))
        f.write(i32(m.mnt_loc)); f.write(f32(m.mnt_m6))
        if len(m.mnt_loc):
            f.write(f32(m.mnt_stf))
        f.write(i32(m.frc_loc)); f.write(f32(m.frc_f3))
        if len(m.frc_loc):
            f.write(f32(m.frc_stf))
        f.write(i32(m.rcv_loc))
        if init_fields is not None:
            for c in range(9):
                f.write(f32(init_fields[c]))
        if _smoothed(m):
            # read by the SrcSmooth build only: moment blocks, then force blocks
            for w, loc in ((m.mnt_smooth, m.mnt_loc), (m.frc_smooth, m.frc_loc)):
                if len(loc):
                    f.write(f32(w))


def _smoothed(m):
    if getattr(m, "foc_smooth", None) is not None:
        raise ValueError("the reference driver takes no focal points")
    return getattr(m, "mnt_smooth", None) is not None or getattr(m, "frc_smooth", None) is not None


def read_output(path, shape):
    n = int(np.prod(shape))
    with open(path, "rb") as f:
        nrecv, nt, nsteps, nstages = struct.unpack("<4i", f.read(16))
        secs = struct.unpack("<d", f.read(8))[0]
        step_secs = np.frombuffer(f.read(8 * nsteps), np.float64).copy()
        seis = np.frombuffer(f.read(9 * nrecv * nt * 4), np.float32).reshape(9, nrecv, nt)
        fw = np.frombuffer(f.read(9 * n * 4), np.float32).reshape(9, *shape)
        w = np.frombuffer(f.read(9 * n * 4), np.float32).reshape(9, *shape)
    return dict(seis=seis.copy(), fw=fw.copy(), w=w.copy(), secs=secs, step_secs=step_secs,
                nsteps=nsteps,
                nstages=nstages)


def run(m, nsteps, init_fields=None, nstages=0, timeout=1800):
    """Runs the reference on the GPU; returns read_output()'s dict."""
    smooth = _smoothed(m)
    if smooth and ((m.mnt_smooth is None and len(m.mnt_loc)) or
                   (m.frc_smooth is None and len(m.frc_loc))):
        raise ValueError("the SrcSmooth build spreads every moment and force")
    binary = REF_BIN_SMOOTH if smooth else REF_BIN
    if not os.path.exists(binary):
        raise FileNotFoundError(f"{binary} not built (make -C {HERE}/ref)")
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        write_input(m, fin, nsteps, init_fields, nstages)
        p = subprocess.run([binary, fin, fout, os.path.join(td, "par")],
                           capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"reference driver failed ({p.returncode}):\n"
                               f"{p.stdout[-2000:]}\n{p.stderr[-2000:]}")
        return read_output(fout, m.shape)
