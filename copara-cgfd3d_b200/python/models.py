"""Synthetic model builders for the CGFD solver (grid, media, CFS-PML,
sources, receivers), in the reference's full-array layout.

The reference reads these from its input files (vmap grid, volume media,
source.dat, station.dat, absorb.dat) that offline MATLAB/Python scripts
write (generatemodel/).  Here the same kinds of models are generated
directly from seeded parameters:

  * flat_halfspace: flat free surface, uniform medium, explosive source,
    surface receivers (the 160x160x80 benchmark model and small test cases);
  * gaussian_hill: Gaussian-hill topography on a hybrid grid (curvilinear
    above the conversion layer ConIndex, Cartesian below) with vertically
    stretched spacing, layered media with a seeded correlated perturbation,
    double-couple source (the 400x400x200 benchmark model and small cases);
  * batch_models: many uneven hill models with random point sources, for the
    batched solver (64 models, sides 96..256, in the default set).

Grid coordinates are extended into the ghost cells by linear extrapolation
(common::interpolated_extend, src/common.cpp:67-95); the metric, CFS-PML
factors, source time functions and moment tensors come from an FP64
pre-processing backend: by default the solver library's
(cgfd.metric_from_coords / cfs_factors / stf / angle2moment); with
use_preprocessing("oracle") the CPU oracle's restatement of the same
reference functions, so that a process which must not load the solver
library (the timing of the reference's own runtime) can still build every
model.  The solver library is imported only when its backend is used or a
solver description is made.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

LFD = 3

# wavelet names of the reference's source.dat (src/source.cpp:723-775)
STF_TYPES = {"Gauss": 0, "gauss": 1, "Ricker": 2, "ricker": 3, "Bell": 4,
             "bell": 5, "BELL": 6, "Step": 7}

_PREP = "product"


def use_preprocessing(backend: str) -> None:
    """Selects the FP64 pre-processing: "product" (libcgfd.so) or "oracle"
    (the CPU oracle's restatement, which never loads libcgfd.so)."""
    global _PREP
    if backend not in ("product", "oracle"):
        raise ValueError(backend)
    _PREP = backend


def _prep():
    if _PREP == "oracle":
        import pyoracle
        return pyoracle
    import cgfd
    return cgfd


def _metric_from_coords(ni, nj, nk, h, x, y, z):
    return _prep().metric_from_coords(ni, nj, nk, h, x, y, z)


def _stf(kind, start, t0, f0, n, dt):
    k = STF_TYPES[kind] if isinstance(kind, str) else int(kind)
    return np.asarray(_prep().stf(k, start, t0, f0, n, dt), np.float32)


def _angle2moment(strike, dip, rake):
    return np.asarray(_prep().angle2moment(strike, dip, rake), np.float64)


@dataclasses.dataclass
class Model:
    name: str
    ni: int
    nj: int
    nk: int
    steph: float
    stept: float
    nt: int
    con_index: int
    nabs: tuple
    metric: dict            # zeta_x zeta_y zeta_z jac, float64 full arrays
    alpha: np.ndarray       # float32 full arrays
    beta: np.ndarray
    rho: np.ndarray
    pml: tuple              # (apd, b, db), each 3 arrays of nx, ny, nz float64
    mnt_loc: np.ndarray     # (n, 3) int32
    mnt_m6: np.ndarray      # (n, 6) float32
    mnt_stf: np.ndarray     # (n, nstf) float32
    frc_loc: np.ndarray
    frc_f3: np.ndarray
    frc_stf: np.ndarray
    rcv_loc: np.ndarray     # (n, 3) int32
    info: dict = dataclasses.field(default_factory=dict)
    # focal (finite-fault) points: (n, 3) int32, moment series [6][n][fnt]
    # float32 sampled every foc_dt seconds from t = 0
    foc_loc: np.ndarray = None
    foc_mom: np.ndarray = None
    foc_dt: float = 0.0
    # source smoothing weights [n][7][7][7] (float64) of the moments, forces
    # and focal points, or None (cgfd_set_source_smoothing)
    mnt_smooth: np.ndarray = None
    frc_smooth: np.ndarray = None
    foc_smooth: np.ndarray = None

    @property
    def cells(self) -> int:
        return self.ni * self.nj * self.nk

    @property
    def shape(self):
        return (self.ni + 6, self.nj + 6, self.nk + 6)

    def desc(self, **kw):
        import cgfd
        return cgfd.make_desc(self.ni, self.nj, self.nk, self.steph, self.stept,
                              self.nt, self.con_index, self.nabs, **kw)

    def load(self, solver):
        """Uploads everything into a solver (cgfd.Solver or the oracle)."""
        m = self.metric
        solver.upload_metric(m["zeta_x"], m["zeta_y"], m["zeta_z"], m["jac"])
        solver.upload_media(self.alpha, self.beta, self.rho)
        solver.upload_pml(*self.pml)
        if len(self.mnt_loc):
            solver.upload_moments(self.mnt_loc, self.mnt_m6, self.mnt_stf)
        if len(self.frc_loc):
            solver.upload_forces(self.frc_loc, self.frc_f3, self.frc_stf)
        if self.foc_loc is not None and len(self.foc_loc):
            solver.upload_focal(self.foc_loc, self.foc_dt, self.foc_mom)
        for kind, w in enumerate((self.mnt_smooth, self.frc_smooth, self.foc_smooth)):
            if w is not None:
                solver.set_source_smoothing(kind, w)
        if len(self.rcv_loc):
            solver.set_receivers(self.rcv_loc)

    def upload_bytes(self) -> int:
        n = int(np.prod(self.shape))
        b = n * 4 * 8 + n * 4 * 3  # metric (4 x f64) + media (3 x f32)
        b += sum(a.nbytes for t in self.pml for a in t)
        b += self.mnt_stf.nbytes + self.frc_stf.nbytes + self.rcv_loc.nbytes
        return b


# ----------------------------------------------------------------------------

def _extend_linear(v: np.ndarray, ni: int, nj: int, nk: int) -> None:
    """common::interpolated_extend: 2*v[edge] - v[edge +- s], Z then Y then X."""
    for s in range(1, LFD + 1):
        v[:, :, LFD - s] = 2.0 * v[:, :, LFD] - v[:, :, LFD + s]
        v[:, :, nk + 2 + s] = 2.0 * v[:, :, nk + 2] - v[:, :, nk + 2 - s]
    for s in range(1, LFD + 1):
        v[:, LFD - s, :] = 2.0 * v[:, LFD, :] - v[:, LFD + s, :]
        v[:, nj + 2 + s, :] = 2.0 * v[:, nj + 2, :] - v[:, nj + 2 - s, :]
    for s in range(1, LFD + 1):
        v[LFD - s, :, :] = 2.0 * v[LFD, :, :] - v[LFD + s, :, :]
        v[ni + 2 + s, :, :] = 2.0 * v[ni + 2, :, :] - v[ni + 2 - s, :, :]


def _zflat(nk: int, dz_top: float, dz_bot: float) -> np.ndarray:
    """Flat stretched z (k index with ghosts); 0 at the surface k = nk+2,
    spacing linear in k from dz_bot (bottom) to dz_top (top)."""
    nint = nk - 1
    if nint > 1:
        sp = dz_bot + (dz_top - dz_bot) * np.arange(nint) / (nint - 1)
    else:
        sp = np.full(nint, dz_top)
    z = np.zeros(nk + 6)
    z[LFD:nk + LFD] = -np.concatenate([np.cumsum(sp[::-1])[::-1], [0.0]])
    return z


def _coords(ni, nj, nk, h, dz_top, dz_bot, hill_h, hill_w, con_index):
    nx, ny, nz = ni + 6, nj + 6, nk + 6
    xc = (np.arange(nx) - LFD - (ni - 1) / 2.0) * h
    yc = (np.arange(ny) - LFD - (nj - 1) / 2.0) * h
    zf = _zflat(nk, dz_top, dz_bot)
    x = np.broadcast_to(xc[:, None, None], (nx, ny, nz)).copy()
    y = np.broadcast_to(yc[None, :, None], (nx, ny, nz)).copy()
    z = np.broadcast_to(zf[None, None, :], (nx, ny, nz)).copy()
    if hill_h != 0.0:
        H = hill_h * np.exp(-(xc[:, None] ** 2 + yc[None, :] ** 2) / hill_w ** 2)
        zc = zf[con_index]
        k = np.arange(con_index, nk + LFD)
        w = (zf[k] - zc) / (0.0 - zc)  # 0 at the conversion layer, 1 at the surface
        z[:, :, con_index:nk + LFD] += H[:, :, None] * w[None, None, :]
    _extend_linear(x, ni, nj, nk)
    _extend_linear(y, ni, nj, nk)
    _extend_linear(z, ni, nj, nk)
    return x, y, z


def _pml(ni, nj, nk, steph, metric, nabs, velabs, bmax, amax):
    def norm(a, b, c):
        n = np.sqrt(a * a + b * b + c * c)
        return np.where(n > 0, steph / np.where(n > 0, n, 1.0), 0.0)
    m = metric
    dlx = norm(m["xi_x"][:, LFD, LFD], m["xi_y"][:, LFD, LFD], m["xi_z"][:, LFD, LFD])
    dly = norm(m["eta_x"][LFD, :, LFD], m["eta_y"][LFD, :, LFD], m["eta_z"][LFD, :, LFD])
    dlz = norm(m["zeta_x"][LFD, LFD, :], m["zeta_y"][LFD, LFD, :], m["zeta_z"][LFD, LFD, :])
    return _prep().cfs_factors(ni, nj, nk, nabs, [velabs] * 6, [bmax] * 6, [amax] * 6,
                            dlx, dly, dlz)


def _solver_metric(metric):
    """The four metric arrays the solver consumes (the rest of calmetric's
    output, xi and eta, is only needed for the PML thicknesses)."""
    return {k: metric[k] for k in ("zeta_x", "zeta_y", "zeta_z", "jac")}


def _surface_grid(ni, nj, n_side, spacing_cells):
    ci, cj = LFD + ni // 2, LFD + nj // 2
    off = (np.arange(n_side) - (n_side - 1) / 2.0) * spacing_cells
    ii = np.rint(ci + off).astype(int)
    jj = np.rint(cj + off).astype(int)
    return np.array([(i, j) for i in ii for j in jj], np.int32)


def flat_halfspace(ni=160, nj=160, nk=80, h=100.0, dt=0.008, nt=500, vp=6000.0,
                   vs=3464.0, rho=2670.0, nabs=(12, 12, 12, 12, 12, 0),
                   src_depth=2000.0, f0=2.0, t0=0.6, n_side=5, rcv_spacing=1000.0,
                   con_depth=3000.0, velabs=8500.0, bmax=2.5, amax=5.0,
                   force=False, name="flat_halfspace") -> Model:
    """Flat free surface, uniform medium, explosive moment source (Ricker),
    surface receivers on an n_side x n_side grid."""
    con_index = max(LFD, nk + LFD - 1 - int(round(con_depth / h)))
    x, y, z = _coords(ni, nj, nk, h, h, h, 0.0, 1.0, con_index)
    metric = _metric_from_coords(ni, nj, nk, h, x, y, z)
    shape = (ni + 6, nj + 6, nk + 6)
    alpha = np.full(shape, vp, np.float32)
    beta = np.full(shape, vs, np.float32)
    dens = np.full(shape, rho, np.float32)
    pml = _pml(ni, nj, nk, h, metric, nabs, velabs, bmax, amax)
    metric = _solver_metric(metric)
    top = nk + LFD - 1
    sk = top - int(round(src_depth / h))
    src = np.array([[LFD + ni // 2, LFD + nj // 2, sk]], np.int32)
    nstf = 2 * (nt + 1)
    wave = _stf("Ricker", 0.0, t0, f0, nstf, dt / 2.0)[None, :]
    m6 = np.array([[1e16, 1e16, 1e16, 0, 0, 0]], np.float32)
    ij = _surface_grid(ni, nj, n_side, rcv_spacing / h)
    rcv = np.concatenate([ij, np.full((len(ij), 1), top, np.int32)], axis=1)
    empty_loc = np.zeros((0, 3), np.int32)
    if force:
        frc_loc = src.copy()
        frc_f3 = np.array([[0.0, 0.0, 1e15]], np.float32)
        frc_stf = wave.copy()
    else:
        frc_loc, frc_f3, frc_stf = empty_loc, np.zeros((0, 3), np.float32), np.zeros((0, nstf), np.float32)
    return Model(name, ni, nj, nk, h, dt, nt, con_index, tuple(nabs), metric, alpha, beta,
                 dens, pml, src, m6, wave.astype(np.float32), frc_loc, frc_f3, frc_stf,
                 rcv.astype(np.int32), info=dict(src_depth=src_depth, f0=f0, t0=t0))


def _gauss_field(shape, corr_cells, rng):
    from scipy.ndimage import gaussian_filter
    f = rng.standard_normal(shape).astype(np.float32)
    f = gaussian_filter(f, sigma=corr_cells, mode="wrap")
    f /= max(float(f.std()), 1e-12)
    return f


def gaussian_hill(ni=400, nj=400, nk=200, h=100.0, dt=0.006, nt=2000,
                  dz_top=50.0, dz_bot=150.0, hill_h=1500.0, hill_w=3000.0,
                  con_depth=3000.0, layers=((-2000.0, 4000.0, 2400.0),
                                            (-8000.0, 5500.0, 2600.0),
                                            (-1e30, 6500.0, 2800.0)),
                  perturb=0.05, corr_len=500.0, seed=12345,
                  nabs=(20, 20, 20, 20, 20, 0), src_depth=5000.0,
                  sdr=(30.0, 60.0, 90.0), m0=1e6, stf_kind="Gauss", f0=0.25,
                  t0=1.0, n_side=20, rcv_spacing=1500.0, velabs=7000.0, bmax=2.5,
                  amax=5.0, force=False, force_f0=2.0, name="gaussian_hill") -> Model:
    """Gaussian-hill topography z = hill_h*exp(-(x^2+y^2)/hill_w^2) on a hybrid
    grid with vertical spacing stretched from dz_top (surface) to dz_bot
    (bottom); layered medium (depth, vp, rho) with vs = vp/sqrt(3) and a
    seeded correlated perturbation; double-couple source (x mu at the source,
    like moment_mech_input = angle); surface receivers."""
    zf = _zflat(nk, dz_top, dz_bot)
    top = nk + LFD - 1
    con_index = int(np.clip(np.searchsorted(zf[LFD:top + 1], -con_depth) + LFD, LFD, top - 3))
    x, y, z = _coords(ni, nj, nk, h, dz_top, dz_bot, hill_h, hill_w, con_index)
    metric = _metric_from_coords(ni, nj, nk, h, x, y, z)
    shape = (ni + 6, nj + 6, nk + 6)
    vp = np.empty(shape, np.float32)
    dens = np.empty(shape, np.float32)
    # layers by depth below the local surface-free reference (z of the flat grid)
    zref = np.broadcast_to(zf[None, None, :], shape)
    vp[...] = layers[-1][1]
    dens[...] = layers[-1][2]
    for zbot, v, r in reversed(layers[:-1]):
        sel = zref > zbot
        vp[sel] = v
        dens[sel] = r
    rng = np.random.default_rng(seed)
    if perturb:
        pert = np.clip(_gauss_field(shape, corr_len / h, rng), -3.0, 3.0) * perturb
        vp *= (1.0 + pert)
        dens *= (1.0 + 0.5 * pert)
        del pert
    vs = (vp / np.float32(math.sqrt(3.0))).astype(np.float32)
    pml = _pml(ni, nj, nk, h, metric, nabs, velabs, bmax, amax)
    metric = _solver_metric(metric)
    ci, cj = LFD + ni // 2, LFD + nj // 2
    sk = int(np.clip(np.searchsorted(zf[LFD:top + 1], -src_depth) + LFD, LFD, top))
    src = np.array([[ci, cj, sk]], np.int32)
    nstf = 2 * (nt + 1)
    wave = _stf(stf_kind, 0.0, t0, f0, nstf, dt / 2.0)[None, :]
    mu = float(dens[ci, cj, sk]) * float(vs[ci, cj, sk]) ** 2
    m6 = (_angle2moment(*sdr) * m0 * mu).astype(np.float32)[None, :]
    ij = _surface_grid(ni, nj, n_side, rcv_spacing / h)
    rcv = np.concatenate([ij, np.full((len(ij), 1), top, np.int32)], axis=1)
    if force:
        frc_loc = np.array([[ci + 2, cj - 1, top]], np.int32)
        frc_f3 = np.array([[3e14, -2e14, 1e15]], np.float32)
        frc_stf = _stf("Ricker", 0.0, t0, force_f0, nstf, dt / 2.0)[None, :]
    else:
        frc_loc = np.zeros((0, 3), np.int32)
        frc_f3 = np.zeros((0, 3), np.float32)
        frc_stf = np.zeros((0, nstf), np.float32)
    return Model(name, ni, nj, nk, h, dt, nt, con_index, tuple(nabs), metric,
                 vp.astype(np.float32), vs, dens.astype(np.float32), pml, src, m6,
                 wave.astype(np.float32), frc_loc, frc_f3, frc_stf.astype(np.float32),
                 rcv.astype(np.int32), info=dict(sdr=sdr, m0=m0, f0=f0, t0=t0))


# ----------------------------- named configs --------------------------------

def config_c1(nt=500) -> Model:
    """160x160x80 flat half-space, h=100 m, vp 6000 / vs 3464 / rho 2670,
    12-cell CFS-PML on 5 faces, explosive Ricker source (f0 2 Hz) at 2 km,
    dt 0.008 s, 25 surface receivers on a 5x5 grid at 1 km spacing."""
    return flat_halfspace(nt=nt, name="flat_halfspace_160x160x80")


def config_c2(nt=2000) -> Model:
    """400x400x200 Gaussian hill (1500 m, width 3000 m), vertical spacing
    50 -> 150 m, 3 layers with 5% perturbation (seed 12345), double couple
    (30/60/90) with a Gaussian STF, 20-cell PML, 400 surface receivers."""
    return gaussian_hill(nt=nt, name="gaussian_hill_400x400x200")


def random_layers(n_layers, depth, vp_range=(2500.0, 7000.0), seed=5):
    """Seeded layered medium for gaussian_hill: n_layers layers with tops at
    sorted uniform depths in (0, 0.9 depth) and vp drawn uniformly from
    vp_range, increasing with depth; density from Gardner's relation
    310 vp^0.25 (kg/m^3, vp in m/s).  Returns ((z_bottom, vp, rho), ...)
    from the top down, the last layer unbounded."""
    rng = np.random.default_rng(seed)
    tops = np.sort(rng.uniform(0.0, 0.9 * depth, n_layers - 1))
    vps = np.sort(rng.uniform(vp_range[0], vp_range[1], n_layers))
    vps[0], vps[-1] = vp_range[0], vp_range[1]
    out = []
    for q in range(n_layers):
        zbot = -float(tops[q]) if q < n_layers - 1 else -1e30
        out.append((zbot, float(vps[q]), float(310.0 * vps[q] ** 0.25)))
    return tuple(out)


def config_c5(nt=3000, nabs=(20, 20, 20, 20, 20, 0), ni=600, nj=600, nk=250,
              name="gaussian_hill_600x600x250", **kw) -> Model:
    """600x600x250 Gaussian hill (the 400x400x200 model's topography: 1500 m,
    width 3000 m, vertical spacing 50 -> 150 m) over a seeded random-layered
    medium (8 layers, vp 2500..7000 increasing with depth, vs = vp/sqrt(3),
    Gardner density), double couple (30/60/90) with a Gaussian STF at 5 km,
    20-cell CFS-PML on the 5 absorbing faces, 400 surface receivers (20 x 20
    at 1.5 km); dt = 7 ms, 0.75 of the reference's bound 1.3 dmin / vp_max
    (src/mediaparas.cpp:2263) with dmin = 50 m and vp_max = 7000 m/s."""
    depth = float(np.sum(np.linspace(50.0, 150.0, nk - 1)))
    return gaussian_hill(ni=ni, nj=nj, nk=nk, dt=0.007, nt=nt,
                         layers=random_layers(8, depth), perturb=0.0, nabs=nabs,
                         velabs=7000.0, name=name, **kw)


def hill_256(nt=40, nabs=(20, 20, 20, 20, 20, 0)) -> Model:
    """The 400x400x200 hill model's generator at 256x256x128 (8.4 M cells,
    about 2 GB on the device): the profiling case for the stage kernels."""
    return gaussian_hill(ni=256, nj=256, nk=128, nt=nt, n_side=5, rcv_spacing=1000.0,
                         nabs=nabs, name="gaussian_hill_256x256x128")


def small_flat(nt=40, ni=28, nj=24, nk=20, **kw) -> Model:
    kw.setdefault("nabs", (5, 5, 5, 5, 5, 0))
    kw.setdefault("src_depth", 600.0)
    return flat_halfspace(ni=ni, nj=nj, nk=nk, h=100.0, dt=0.008, nt=nt,
                          f0=4.0, t0=0.3, n_side=3,
                          rcv_spacing=400.0, con_depth=800.0, name="small_flat", **kw)


def small_hill(nt=40, ni=30, nj=26, nk=22, seed=7, **kw) -> Model:
    kw.setdefault("nabs", (5, 6, 4, 5, 5, 0))
    return gaussian_hill(ni=ni, nj=nj, nk=nk, h=100.0, dt=0.006, nt=nt, dz_top=60.0,
                         dz_bot=120.0, hill_h=400.0, hill_w=800.0, con_depth=900.0,
                         layers=((-500.0, 4000.0, 2400.0), (-1200.0, 5500.0, 2600.0),
                                 (-1e30, 6500.0, 2800.0)),
                         corr_len=200.0, seed=seed, src_depth=900.0, f0=0.08,
                         t0=0.25, n_side=3, rcv_spacing=500.0, velabs=7000.0,
                         name="small_hill", **kw)


def batch_models(n=64, seed=7, nt=1000, side=(96, 256), nabs_cells=12, h=100.0,
                 name="batch") -> list:
    """n independent models of uneven size for a batch: sides U{96..256}
    (nz = side/2), Gaussian hill height U(0, 2000) m and width U(1, 5) km,
    two layers with vp U(3000, 7000) and vs = vp/1.73 (density 2600/2800), a
    random point moment source (M_ij ~ N(0, 1) x 1e15) with a Ricker STF of
    f0 U(1, 4) Hz, 5 x 5 surface receivers, 12-cell CFS-PML, dt at 0.8 of
    the reference's stability bound 1.3 dmin / vp_max (src/mediaparas.cpp:2263;
    dmin = the top vertical spacing, the smallest of the grid); seeded."""
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        s = int(rng.integers(side[0], side[1] + 1))
        nk = s // 2
        hill_h = float(rng.uniform(0.0, 2000.0))
        hill_w = float(rng.uniform(1000.0, 5000.0))
        vp1, vp2 = sorted(rng.uniform(3000.0, 7000.0, 2))
        dz_top, dz_bot = 0.5 * h, 1.5 * h
        dt = 0.8 * 1.3 * min(dz_top, h) / max(vp1, vp2)
        f0 = float(rng.uniform(1.0, 4.0))
        depth = nk * h
        m = gaussian_hill(ni=s, nj=s, nk=nk, h=h, dt=dt, nt=nt, dz_top=dz_top, dz_bot=dz_bot,
                          hill_h=hill_h, hill_w=hill_w, con_depth=min(3000.0, 0.3 * depth),
                          layers=((-0.3 * depth, vp1, 2600.0), (-1e30, vp2, 2800.0)),
                          perturb=0.0, nabs=(nabs_cells,) * 5 + (0,),
                          src_depth=float(rng.uniform(0.2, 0.5)) * depth, stf_kind="Ricker",
                          f0=f0, t0=1.2 / f0, n_side=5, rcv_spacing=0.1 * s * h,
                          velabs=1.2 * max(vp1, vp2), name=f"{name}_{q}")
        m6 = (rng.standard_normal(6) * 1e15).astype(np.float32)[None, :]
        m = dataclasses.replace(m, mnt_m6=m6, info=dict(m.info, f0=f0, vp=(vp1, vp2)))
        out.append(m)
    return out


def gaussian_blocks(n, seed, top_rows=None):
    """n smoothing blocks [n][7][7][7] shaped like the reference's SrcSmooth
    weights: exp(-(offset - shift)^2 / 1.5^2) per axis around a seeded
    sub-cell shift in [-1/2, 1/2), normalised to 1 (top_rows[q] < 7: over
    the first top_rows[q] z-rows only, the rows at or below the surface)."""
    rng = np.random.default_rng(seed)
    o = np.arange(-3, 4, dtype=np.float64)
    out = np.zeros((n, 7, 7, 7))
    for q in range(n):
        sh = rng.uniform(-0.5, 0.5, 3)
        g = [np.exp(-(o - s) ** 2 / 2.25) for s in sh]
        w = g[0][:, None, None] * g[1][None, :, None] * g[2][None, None, :]
        w /= w.sum()
        if top_rows is not None and top_rows[q] < 7:
            w /= w[:, :, :top_rows[q]].sum()
        out[q] = w
    return out


def small_hill_smoothed(nt=60, seed=21) -> Model:
    """small_hill with its surface force and a second moment two cells from
    the x- side (its block crosses the side), all sources spread over 7^3
    nodes with gaussian_blocks (the force's block crosses the surface)."""
    m = small_hill(nt=nt, force=True)
    loc = np.concatenate([m.mnt_loc, [[5, 3 + m.nj // 3, 3 + m.nk - 8]]]).astype(np.int32)
    m6 = np.concatenate([m.mnt_m6, 0.5 * m.mnt_m6[:, ::-1]]).astype(np.float32)
    stf = np.concatenate([m.mnt_stf, m.mnt_stf]).astype(np.float32)
    top = m.nk + LFD - 1
    wm = gaussian_blocks(len(loc), seed)
    wf = gaussian_blocks(len(m.frc_loc), seed + 1, [top + 1 - k + 3 for k in m.frc_loc[:, 2]])
    return dataclasses.replace(m, name="small_hill_smoothed", mnt_loc=loc, mnt_m6=m6,
                               mnt_stf=stf, mnt_smooth=wm, frc_smooth=wf)


def with_finite_fault(m: Model, center, length=8, width=5, strike=30.0, dip=60.0, rake=90.0,
                      m0=1e15, vr=2500.0, rise=0.4, fdt=None, seed=3) -> Model:
    """Adds a planar finite fault of length x width points (one per cell on a
    grid of h spacing along strike and down dip) centred at the reference
    index `center`: a rupture spreading from the centre at speed vr, each
    point's moment rate a triangle of duration `rise` scaled by a random
    slip weight (seed), the mechanism (strike, dip, rake) from angle2moment,
    the series sampled every fdt (default 1.7 * stept, which is not a
    multiple of the half step, so stage times fall between samples)."""
    rng = np.random.default_rng(seed)
    h = m.steph
    fdt = fdt or 1.7 * m.stept
    m6 = np.asarray(_angle2moment(strike, dip, rake), np.float64)
    st, dp = math.radians(strike), math.radians(dip)
    sv = np.array([math.sin(st), math.cos(st), 0.0])              # along strike (x east, y north)
    dv = np.array([math.cos(dp) * math.cos(st), -math.cos(dp) * math.sin(st), -math.sin(dp)])
    pts, dist = [], []
    for a in range(length):
        for b in range(width):
            sa, db = (a - (length - 1) / 2) * h, (b - (width - 1) / 2) * h
            p = np.array(center, np.float64) + (sa * sv + db * dv) / h
            pts.append(np.rint(p).astype(np.int32))
            dist.append(math.hypot(sa, db))
    loc = np.array(pts, np.int32)
    n = len(loc)
    t_end = max(dist) / vr + rise
    fnt = int(math.ceil(t_end / fdt)) + 3
    t = np.arange(fnt) * fdt
    w = rng.uniform(0.5, 1.5, n)
    w *= 1.0 / w.sum()
    mom = np.zeros((6, n, fnt), np.float32)
    for q in range(n):
        t0 = dist[q] / vr
        tri = np.clip(1.0 - np.abs(t - t0 - rise / 2) / (rise / 2), 0.0, None) * (2.0 / rise)
        for c in range(6):
            mom[c, q] = m0 * w[q] * m6[c] * tri
    return dataclasses.replace(m, foc_loc=loc, foc_mom=mom, foc_dt=float(fdt))
