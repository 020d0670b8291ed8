"""Shared helpers for the tests (comparison metrics, model runs)."""
import numpy as np


def rel_l2(a, b):
    """||a - b|| / ||b|| over all entries (b is the reference)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))


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
