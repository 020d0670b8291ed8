"""Parity cases shared by the GPU tests, the golden-vector generator and the
CPU golden tests.  Every case is rebuilt deterministically from its seeded
parameters; model_digest() pins the inputs a golden file was made from."""
import hashlib

import numpy as np

import models

# name -> (builder, kwargs, full steps, partial stages, random initial field seed)
CASES = {
    "flat_60": (models.small_flat, dict(nt=60), 60, 0, None),
    "flat_force_60": (models.small_flat, dict(nt=60, force=True), 60, 0, None),
    "hill_60": (models.small_hill, dict(nt=60, force=True), 60, 0, None),
    "hill_stage1": (models.small_hill, dict(nt=8, ni=18, nj=16, nk=14, nabs=(3, 4, 3, 3, 4, 0)), 0, 1, 11),
    "hill_stage4": (models.small_hill, dict(nt=8, ni=18, nj=16, nk=14, nabs=(3, 4, 3, 3, 4, 0)), 0, 4, 12),
    "hill_step5": (models.small_hill, dict(nt=8, ni=18, nj=16, nk=14, nabs=(3, 4, 3, 3, 4, 0)), 5, 2, 13),
    # moments and a surface force spread over 7^3 nodes (the SrcSmooth build)
    "hill_smooth_60": (models.small_hill_smoothed, dict(nt=60), 60, 0, None),
}


def build(name):
    b, kw, nsteps, nstages, seed = CASES[name]
    m = b(**kw)
    init = random_fields(m, seed) if seed is not None else None
    return m, nsteps, nstages, init


def random_fields(m, seed):
    """Smooth random wavefield (valid cells only) with velocity ~1 m/s and
    stress ~1e7 Pa, so every stencil term is exercised at realistic scale."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    out = np.zeros((9,) + m.shape, np.float32)
    for c in range(9):
        f = gaussian_filter(rng.standard_normal(m.shape), 1.2, mode="wrap")
        f /= f.std()
        out[c][3:-3, 3:-3, 3:-3] = f[3:-3, 3:-3, 3:-3] * (1.0 if c < 3 else 1e7)
    return out


def model_digest(m, init=None):
    h = hashlib.sha256()
    for k in ("zeta_x", "zeta_y", "zeta_z", "jac"):
        h.update(np.ascontiguousarray(m.metric[k], np.float32).tobytes())
    for a in (m.alpha, m.beta, m.rho, m.mnt_loc, m.mnt_m6, m.mnt_stf, m.frc_loc,
              m.frc_f3, m.frc_stf, m.rcv_loc):
        h.update(np.ascontiguousarray(a).tobytes())
    for g in m.pml:
        for a in g:
            h.update(np.ascontiguousarray(a, np.float32).tobytes())
    for w in (m.mnt_smooth, m.frc_smooth):
        if w is not None:
            h.update(np.ascontiguousarray(w, np.float32).tobytes())
    if m.foc_loc is not None and len(m.foc_loc):
        h.update(np.ascontiguousarray(m.foc_loc, np.int32).tobytes())
        h.update(np.ascontiguousarray(m.foc_mom, np.float32).tobytes())
        h.update(np.float64(m.foc_dt).tobytes())
    if init is not None:
        h.update(np.ascontiguousarray(init).tobytes())
    return h.hexdigest()


def run_oracle(m, nsteps, nstages, init, prec=0):
    """Runs the CPU oracle like the reference driver: nsteps full steps, then
    nstages stages of the next step.  Returns (seis, FW, W)."""
    import pyoracle
    DIRS = [[(1, 1, 1), (-1, -1, -1), (1, 1, 1), (-1, -1, -1)],
            [(1, 1, -1), (-1, -1, 1), (1, 1, -1), (-1, -1, 1)],
            [(-1, -1, -1), (1, 1, 1), (-1, -1, -1), (1, 1, 1)],
            [(-1, -1, 1), (1, 1, -1), (-1, -1, 1), (1, 1, -1)]]
    o = pyoracle.OracleSolver(m.desc(), prec)
    m.load(o)
    if init is not None:
        for c in range(9):
            o.set_field(c, init[c])
    o.step(nsteps)
    for s in range(nstages):
        o.rk_stage(s, nsteps, *DIRS[nsteps % 4][s])
    seis = o.seismograms()
    fw = np.stack([o.get_field(c, 0) for c in range(9)])
    w = np.stack([o.get_field(c, 1) for c in range(9)])
    o.close()
    return seis, fw, w


def run_product(m, nsteps, nstages, init, kernel=None):
    import cgfd
    DIRS = [[(1, 1, 1), (-1, -1, -1), (1, 1, 1), (-1, -1, -1)],
            [(1, 1, -1), (-1, -1, 1), (1, 1, -1), (-1, -1, 1)],
            [(-1, -1, -1), (1, 1, 1), (-1, -1, -1), (1, 1, 1)],
            [(-1, -1, 1), (1, 1, -1), (-1, -1, 1), (1, 1, -1)]]
    kw = {} if kernel is None else dict(kernel=kernel)
    s = cgfd.Solver(m.desc(**kw))
    m.load(s)
    if init is not None:
        for c in range(9):
            s.set_field(c, init[c])
    s.step(nsteps)
    for st in range(nstages):
        s.rk_stage(st, nsteps, *DIRS[nsteps % 4][st])
    seis = s.seismograms()
    fw = np.stack([s.get_field(c, cgfd.SET_FW) for c in range(9)])
    w = np.stack([s.get_field(c, cgfd.SET_W) for c in range(9)])
    s.close()
    return seis, fw, w


# ---- the reference's other outputs and its focal source (one case) ----------
# A 24-point finite fault on the small hill (one point per cell: the
# reference's LoadRmom adds from one thread per point without atomics, so
# points sharing a cell race there), peak velocity on, and snapshots of a
# strided sub-volume of all nine components every SNAP_TINV steps.
OUTPUT_CASE = "outputs_focal_pv_snap_36"
SNAP_START, SNAP_COUNT, SNAP_STRIDE, SNAP_TINV = (4, 5, 6), (8, 6, 5), (3, 3, 3), 4


def build_outputs_case(nt=36):
    import dataclasses
    m = models.small_hill(nt=nt, nabs=(5, 6, 4, 5, 5, 0))
    m = dataclasses.replace(m, mnt_loc=np.zeros((0, 3), np.int32),
                            mnt_m6=np.zeros((0, 6), np.float32),
                            mnt_stf=np.zeros((0, m.mnt_stf.shape[1]), np.float32))
    m = models.with_finite_fault(m, center=(3 + m.ni // 2, 3 + m.nj // 2, 3 + m.nk - 9),
                                 length=6, width=4, m0=1e15, vr=2500.0, rise=0.06)
    _, first = np.unique(m.foc_loc, axis=0, return_index=True)
    keep = np.sort(first)
    return dataclasses.replace(m, foc_loc=np.ascontiguousarray(m.foc_loc[keep]),
                               foc_mom=np.ascontiguousarray(m.foc_mom[:, keep]))


def snap_points():
    """The snapshot points in [i][j][k] order (reference full-array indices)."""
    ax = [s + d * np.arange(n) for s, n, d in zip(SNAP_START, SNAP_COUNT, SNAP_STRIDE)]
    g = np.meshgrid(*ax, indexing="ij")
    return np.stack([a.reshape(-1) for a in g], axis=1).astype(np.int32)


def run_oracle_outputs(m, nsteps):
    """The oracle stepped one step at a time: seismograms, the peak |V| of
    the top valid layer over the steps ([3][ni][nj], as IterationFinalPV
    keeps it) and the snapshot samples ([9][point][time index], as SWpick
    takes them from FW after every SNAP_TINV-th step)."""
    import pyoracle
    o = pyoracle.OracleSolver(m.desc(), 0)
    m.load(o)
    top = m.nk + 2
    pv = np.zeros((3, m.ni, m.nj))
    pts = snap_points()
    ntime = (m.nt + SNAP_TINV - 1) // SNAP_TINV
    snap = np.zeros((9, len(pts), ntime))
    for t in range(nsteps):
        o.step(1)
        f = [o.get_field(c, 0) for c in range(9)]
        for c in range(3):
            pv[c] = np.maximum(pv[c], np.abs(f[c][3:-3, 3:-3, top]))
        if t % SNAP_TINV == 0:
            for c in range(9):
                snap[c, :, t // SNAP_TINV] = f[c][pts[:, 0], pts[:, 1], pts[:, 2]]
    seis = o.seismograms()
    o.close()
    return seis, pv, snap
