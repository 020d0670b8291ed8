"""GPU parity: the B200 solver against the FP64 CPU oracle and against the
reference's own CUDA device runtime (oracle/_ref/ref_wavesim, built from the
reference's src/calculate.cu) on the same inputs.

Tolerances: seismograms and fields within 1e-5 relative L2 of the reference
(the parity bar for FP32 arithmetic), and within 1e-5 of the FP64 oracle for
these short runs.
"""
import numpy as np
import pytest

import cases
import cgfd
import refio
from helpers import comp_errors, rel_l2, valid

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _cmp(a, b, tol, what):
    for c, e in enumerate(comp_errors(a, b)):
        assert e < tol, f"{what} component {cgfd.COMPONENTS[c]}: rel L2 {e:.3e}"


KERNELS = [cgfd.KERNEL_SIMPLE, cgfd.KERNEL_FUSED, cgfd.KERNEL_SCALAR]
KIDS = ["simple", "fused", "scalar"]


def _skip_if_unsupported(kernel, m):
    try:
        cgfd.Solver(m.desc(kernel=kernel)).close()
    except cgfd.CgfdError as e:
        if kernel != cgfd.KERNEL_SIMPLE and "kernel does not support" in str(e):
            pytest.skip("tiled kernel not built for this grid")
        raise


@pytest.mark.parametrize("kernel", KERNELS, ids=KIDS)
@pytest.mark.parametrize("name", list(cases.CASES))
def test_product_matches_fp64_oracle(name, kernel):
    m, nsteps, nstages, init = cases.build(name)
    _skip_if_unsupported(kernel, m)
    ps, pfw, pw = cases.run_product(m, nsteps, nstages, init, kernel=kernel)
    os_, ofw, ow = cases.run_oracle(m, nsteps, nstages, init)
    if nsteps:
        _cmp(ps, os_, TOL, "seismogram")
    _cmp(valid(pw), valid(ow), TOL, "W")
    if nstages < 4:
        _cmp(valid(pfw), valid(ofw), TOL, "FW")


@pytest.mark.parametrize("name", list(cases.CASES))
def test_reference_matches_fp64_oracle(name):
    """Pins the oracle to the reference's own CUDA path."""
    m, nsteps, nstages, init = cases.build(name)
    r = refio.run(m, nsteps, init, nstages)
    os_, ofw, ow = cases.run_oracle(m, nsteps, nstages, init)
    if nsteps:
        _cmp(r["seis"], os_, TOL, "seismogram")
    _cmp(valid(r["w"]), valid(ow), TOL, "W")
    if nstages < 4:
        _cmp(valid(r["fw"]), valid(ofw), TOL, "FW")


@pytest.mark.parametrize("kernel", KERNELS, ids=KIDS)
@pytest.mark.parametrize("name", list(cases.CASES))
def test_product_matches_reference(name, kernel):
    m, nsteps, nstages, init = cases.build(name)
    _skip_if_unsupported(kernel, m)
    r = refio.run(m, nsteps, init, nstages)
    ps, pfw, pw = cases.run_product(m, nsteps, nstages, init, kernel=kernel)
    if nsteps:
        _cmp(ps, r["seis"], TOL, "seismogram")
    _cmp(valid(pw), valid(r["w"]), TOL, "W")
    if nstages < 4:
        _cmp(valid(pfw), valid(r["fw"]), TOL, "FW")


@pytest.mark.parametrize("kernel", KERNELS, ids=KIDS)
def test_flat_halfspace_160x160x80_500_steps_matches_reference(kernel):
    """The 160x160x80 flat half-space model, full 500 steps, 25 receivers."""
    import models
    m = models.config_c1()
    _skip_if_unsupported(kernel, m)
    r = refio.run(m, m.nt)
    s = cgfd.Solver(m.desc(kernel=kernel))
    m.load(s)
    s.step(m.nt)
    ps = s.seismograms()
    s.close()
    # the velocity seismograms strictly, per component
    for c in range(3):
        e = rel_l2(ps[c], r["seis"][c])
        assert e < TOL, f"{cgfd.COMPONENTS[c]} rel L2 {e:.3e}"
    _cmp(ps, r["seis"], TOL, "seismogram")


def test_tiled_kernels_match_simple_kernel_on_hill_400x400x200():
    """Full-size property check on the 400x400x200 hill model: 8 steps of the
    tiled kernels (many work items per persistent CTA) against the untiled
    per-cell kernel, seismograms and the final wavefield."""
    import models
    m = models.config_c2(nt=8)
    out = {}
    for kern in KERNELS:
        s = cgfd.Solver(m.desc(kernel=kern))
        m.load(s)
        s.step(8)
        fw = np.stack([s.get_field(c)[::3, ::3, 3:-3] for c in range(9)])
        out[kern] = (s.seismograms(), fw)
        s.close()
    ref = out[cgfd.KERNEL_SIMPLE]
    for kern in (cgfd.KERNEL_FUSED, cgfd.KERNEL_SCALAR):
        for c, e in enumerate(comp_errors(out[kern][1], ref[1])):
            assert e < 1e-5, (kern, cgfd.COMPONENTS[c], e)
        for c, e in enumerate(comp_errors(out[kern][0], ref[0])):
            assert e < 1e-5, (kern, cgfd.COMPONENTS[c], e)


@pytest.mark.parametrize("nstages", [1, 2, 3])
def test_rk_accumulator_between_stages_matches_fp64_oracle(nstages):
    """The default kernels skip tW in the first stage and
    rebuild them in the second from FW and the first stage's output; driven
    stage by stage, tW is materialised after the first stage.  tW after 1, 2
    and 3 stages, and W after them, against the oracle (PML on five faces,
    a moment and a force source)."""
    import pyoracle
    m, _, _, init = cases.build("hill_stage4")
    dirs = [(1, 1, 1), (-1, -1, -1), (1, 1, 1)]
    p = cgfd.Solver(m.desc(kernel=cgfd.KERNEL_FUSED))
    o = pyoracle.OracleSolver(m.desc(), 0)
    for s in (p, o):
        m.load(s)
        for c in range(9):
            s.set_field(c, init[c])
        for st in range(nstages):
            s.rk_stage(st, 0, *dirs[st])
    for fset, what in ((cgfd.SET_TW, "tW"), (cgfd.SET_W, "W")):
        got = np.stack([p.get_field(c, fset) for c in range(9)])
        ref = np.stack([o.get_field(c, fset) for c in range(9)])
        _cmp(valid(got), valid(ref), TOL, f"{what} after {nstages} stage(s)")
    p.close()
    o.close()


def test_shifted_tile_grid_matches_fp64_oracle():
    """A 200-cell-wide model with 10-cell x layers: the paired kernels'
    tile grid then starts at i = -32 (fewer columns in x-layer tiles at the
    same tile-column count), so tiles reach left of the grid and their boxes
    start at negative x.  Seismograms and fields against the oracle."""
    import models
    m = models.small_hill(nt=40, ni=200, nj=20, nk=16, nabs=(10, 10, 5, 5, 5, 0))
    init = cases.random_fields(m, 21)  # every tile active from the first step
    steps = 30
    ps, pfw, _ = cases.run_product(m, steps, 0, init, kernel=cgfd.KERNEL_FUSED)
    os_, ofw, _ = cases.run_oracle(m, steps, 0, init)
    assert np.abs(os_[:3]).max() > 0
    _cmp(ps, os_, TOL, "seismogram")
    _cmp(valid(pfw), valid(ofw), TOL, "FW")


def test_upload_checks_on_converted_values():
    """The metric and media checks run inside the conversion pass: a flat
    model takes the flat path, a hill the per-plane zeta_z table, and a
    non-positive density on one valid cell is refused and leaves the solver
    without media (stepping is refused until valid media arrive)."""
    for name in ("flat_60", "hill_60"):
        m, nsteps, nstages, init = cases.build(name)
        ps, _, _ = cases.run_product(m, 6, 0, init)
        os_, _, _ = cases.run_oracle(m, 6, 0, init)
        _cmp(ps[:, :, :6], os_[:, :, :6], TOL, "seismogram")
    m, _, _, _ = cases.build("hill_60")
    s = cgfd.Solver(m.desc())
    m.load(s)
    rho = m.rho.copy()
    rho[3 + m.ni // 2, 3 + m.nj // 3, 3 + m.nk // 2] = 0.0
    with pytest.raises(cgfd.CgfdError, match="non-positive density"):
        s.upload_media(m.alpha, m.beta, rho)
    with pytest.raises(cgfd.CgfdError):
        s.step(1)
    s.upload_media(m.alpha, m.beta, m.rho)
    s.step(2)
    s.close()
