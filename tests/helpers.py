"""Shared helpers for the tests (comparison metrics, model runs)."""
import numpy as np


def rel_l2(a, b):
    """||a - b|| / ||b|| over all entries (b is the reference)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))


FLOOR = 1e-2


def comp_errors(a, b, floor=FLOOR):
    """Per-component relative L2 error of a against the reference b, arrays
    shaped (9, ...) in Vx Vy Vz Txx Tyy Tzz Txy Txz Tyz order.  Each component
    is normalised by max(||b_c||, floor * max ||b|| over its group) (floor 1e-2:
    an error of 1e-5 on that scale is 1e-7 of the group, FP32 resolution), the
    groups being the velocities and the stresses: a component that vanishes
    in exact arithmetic (the normal traction Tzz, Txz, Tyz at a flat free
    surface, which the reference holds at FP32 round-off, ~1e-8 of the stress
    scale) is then measured on the scale of its group instead of on its own
    round-off."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    norms = [np.linalg.norm(b[c]) for c in range(9)]
    out = []
    for c in range(9):
        grp = norms[0:3] if c < 3 else norms[3:9]
        den = max(norms[c], floor * max(grp))
        d = np.linalg.norm(a[c] - b[c])
        out.append(float(d / den) if den > 0 else float(d))
    return out


def seis_rel_l2(a, b, comps=(0, 1, 2)):
    """Per-component relative L2 of seismograms shaped (9, nrecv, nt)."""
    return [rel_l2(a[c], b[c]) for c in comps]


def valid(f):
    """Valid-cell view of a full (nx, ny, nz) array."""
    return f[..., 3:-3, 3:-3, 3:-3]


def run_solver(solver, model, nsteps):
    model.load(solver)
    solver.step(nsteps)
    return solver.seismograms()
