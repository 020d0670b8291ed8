"""Input/output of the reference parity driver (oracle/_ref/ref_wavesim).

TEST INFRASTRUCTURE ONLY.  write_input() serialises a model (the same arrays
that feed cgfd.Solver and the CPU oracle); run() executes the reference's own
ChildProcs time loop on the GPU (built by oracle/ref/Makefile from the
reference's sources); the result holds its seismograms (HPW layout) and, as
asked, the final FW and W fields, the peak velocities and snapshot samples.
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
# the same runtime built as the reference ships it (-arch=sm_60 -G)
REF_BIN_SHIPPED = os.path.join(HERE, "_ref", "ref_wavesim_shipped")
MAGIC = 0x52464743


def available() -> bool:
    return os.path.exists(REF_BIN)


def write_input(m, path, nsteps, init_fields=None, nstages=0, fields=True, focal=False,
                peak_velocity=False, snap_points=None, snap_tinv=1):
    """Format version 2: a 28-word header, steph/stept/fdt, the model, then
    the optional initial fields, focal points (focal=True: m.foc_loc and
    m.foc_mom [6][n][fnt] sampled every m.foc_dt), snapshot points
    (snap_points (n, 3), all nine components every snap_tinv steps) and the
    SrcSmooth blocks.  fields=False skips the final FW/W dump (benchmark
    sizes)."""
    nstf = m.mnt_stf.shape[1] if len(m.mnt_loc) else (m.frc_stf.shape[1] if len(m.frc_loc) else 0)
    if len(m.mnt_loc) and len(m.frc_loc) and m.mnt_stf.shape[1] != m.frc_stf.shape[1]:
        raise ValueError("moment and force STFs must have the same length")
    nfoc = len(m.foc_loc) if focal and m.foc_loc is not None else 0
    fnt = int(m.foc_mom.shape[-1]) if nfoc else 0
    snap = (np.zeros((0, 3), np.int32) if snap_points is None
            else np.ascontiguousarray(snap_points, np.int32).reshape(-1, 3))
    hdr = [MAGIC, 2, m.ni, m.nj, m.nk, m.nt, nsteps, m.con_index, *m.nabs,
           len(m.mnt_loc), len(m.frc_loc), nstf, len(m.rcv_loc),
           1 if init_fields is not None else 0, nstages, 1 if fields else 0,
           nfoc, fnt, 1 if peak_velocity else 0, len(snap), int(snap_tinv), 0, 0]
    f32 = lambda a: np.ascontiguousarray(a, np.float32).tobytes()
    i32 = lambda a: np.ascontiguousarray(a, np.int32).tobytes()
    with open(path, "wb") as f:
        f.write(struct.pack("<28i", *hdr))
        f.write(struct.pack("<3d", m.steph, m.stept, float(m.foc_dt) if nfoc else 0.0))
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
        if nfoc:
            f.write(i32(m.foc_loc))
            f.write(f32(np.asarray(m.foc_mom, np.float32).reshape(6, nfoc, fnt)))
        if len(snap):
            f.write(i32(snap))
        if _smoothed(m):
            # read by the SrcSmooth build only: moment blocks, then force blocks
            for w, loc in ((m.mnt_smooth, m.mnt_loc), (m.frc_smooth, m.frc_loc)):
                if len(loc):
                    f.write(f32(w))


def _smoothed(m):
    return getattr(m, "mnt_smooth", None) is not None or getattr(m, "frc_smooth", None) is not None


def read_output(path, shape, fields=True, peak_velocity=False, nsnap=0, snap_tinv=1):
    n = int(np.prod(shape))
    out = {}
    with open(path, "rb") as f:
        nrecv, nt, nsteps, nstages = struct.unpack("<4i", f.read(16))
        secs = struct.unpack("<d", f.read(8))[0]
        step_secs = np.frombuffer(f.read(8 * nsteps), np.float64).copy()
        seis = np.frombuffer(f.read(9 * nrecv * nt * 4), np.float32).reshape(9, nrecv, nt)
        if fields:
            out["fw"] = np.frombuffer(f.read(9 * n * 4), np.float32).reshape(9, *shape).copy()
            out["w"] = np.frombuffer(f.read(9 * n * 4), np.float32).reshape(9, *shape).copy()
        if peak_velocity:
            n2 = shape[0] * shape[1]
            out["pv"] = np.frombuffer(f.read(3 * n2 * 4), np.float32).reshape(
                3, shape[0], shape[1]).copy()
        if nsnap:
            ntime = (nt + snap_tinv - 1) // snap_tinv
            out["snap"] = np.frombuffer(f.read(9 * nsnap * ntime * 4), np.float32).reshape(
                9, nsnap, ntime).copy()
    out.update(seis=seis.copy(), secs=secs, step_secs=step_secs, nsteps=nsteps,
               nstages=nstages)
    return out


def run(m, nsteps, init_fields=None, nstages=0, timeout=1800, fields=True, focal=False,
        peak_velocity=False, snap_points=None, snap_tinv=1, binary=None):
    """Runs the reference on the GPU; returns read_output()'s dict: the
    seismograms (HPW), the step times, and as asked the final FW and W
    fields, the peak velocities (Dpv, [3][nx][ny]) and the snapshot samples
    (HSW, [9][point][time index])."""
    smooth = _smoothed(m)
    if smooth and ((m.mnt_smooth is None and len(m.mnt_loc)) or
                   (m.frc_smooth is None and len(m.frc_loc))):
        raise ValueError("the SrcSmooth build spreads every moment and force")
    if focal and getattr(m, "foc_smooth", None) is not None:
        raise ValueError("the driver takes focal points without smoothing")
    if binary is None:
        binary = REF_BIN_SMOOTH if smooth else REF_BIN
    elif smooth:
        raise ValueError("smoothed sources need the SrcSmooth build")
    if not os.path.exists(binary):
        raise FileNotFoundError(f"{binary} not built (make -C {HERE}/ref)")
    nsnap = 0 if snap_points is None else len(np.asarray(snap_points).reshape(-1, 3))
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        write_input(m, fin, nsteps, init_fields, nstages, fields, focal, peak_velocity,
                    snap_points, snap_tinv)
        p = subprocess.run([binary, fin, fout, os.path.join(td, "par")],
                           capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"reference driver failed ({p.returncode}):\n"
                               f"{p.stdout[-2000:]}\n{p.stderr[-2000:]}")
        return read_output(fout, m.shape, fields, peak_velocity, nsnap, snap_tinv)
