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
