"""cgfd_media_volume (the reference's volume media path) against the CPU
restatement (oracle/media_oracle.py, written independently) and exact
cases: a volume linear in x, y, z is reproduced at every valid node inside
it, sub-cell averaging (harmonic lambda and mu, arithmetic density) where
Vp jumps, a fluid layer, the ghost-node fill and the input checks.  The
reference's mediaparas.cpp does not compile with this image's g++, so no
fixture from the reference itself pins this path."""
import glob
import os

import numpy as np
import pytest

import cgfd
import media_oracle as MO

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _grid(name="grid_vmap_hybrid_graded"):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    return g["x"], g["y"], g["z"], int(g["ni"]), int(g["nj"]), int(g["nk"])


def _axes(x, y, z, nv=(9, 8, 12), pad=150.0):
    V = slice(3, -3)
    return [np.linspace(c[V, V, V].min() - pad, c[V, V, V].max() + pad, n)
            for c, n in zip((x, y, z), nv)]


def test_linear_volume_is_reproduced_exactly():
    x, y, z, ni, nj, nk = _grid()
    vx, vy, vz = _axes(x, y, z)
    X, Y, Z = np.meshgrid(vx, vy, vz, indexing="ij")
    vp = (5000.0 + 0.1 * X - 0.05 * Y - 0.2 * Z).astype(np.float32)
    vs = (vp / np.float32(1.8)).astype(np.float32)
    rho = (2500.0 + 0.01 * X + 0.02 * Y).astype(np.float32)
    a, b, r = cgfd.media_volume(x, y, z, vx, vy, vz, vp, vs, rho)
    V = slice(3, -3)
    xv, yv, zv = x[V, V, V], y[V, V, V], z[V, V, V]
    # trilinear interpolation reproduces a linear field (vp, rho as FP32 inputs)
    assert np.allclose(a[V, V, V], 5000.0 + 0.1 * xv - 0.05 * yv - 0.2 * zv, rtol=2e-6)
    assert np.allclose(r[V, V, V], 2500.0 + 0.01 * xv + 0.02 * yv, rtol=2e-6)
    assert np.allclose(b[V, V, V], a[V, V, V] / 1.8, rtol=2e-6)


@pytest.mark.parametrize("samp", [(1, 1, 1), (2, 2, 2), (3, 1, 2)])
def test_layered_volume_matches_restatement(samp):
    x, y, z, ni, nj, nk = _grid()
    vx, vy, vz = _axes(x, y, z)
    rng = np.random.default_rng(5)
    X, Y, Z = np.meshgrid(vx, vy, vz, indexing="ij")
    vp = np.where(Z > -1500.0, 3000.0, 5500.0) + rng.normal(0, 30.0, X.shape)
    vs = vp / np.sqrt(3.0)
    rho = np.where(Z > -1500.0, 2200.0, 2700.0) + rng.normal(0, 10.0, X.shape)
    vp, vs, rho = (v.astype(np.float32) for v in (vp, vs, rho))
    got = cgfd.media_volume(x, y, z, vx, vy, vz, vp, vs, rho, 100.0, 0.1, samp)
    ref = MO.media_volume(x, y, z, ni, nj, nk, vx, vy, vz, vp, vs, rho, 100.0, 0.1, samp)
    for gq, rq in zip(got, ref):
        assert np.abs(gq - rq).max() <= 1e-6 * np.abs(rq).max()
    if max(samp) > 1:  # the jump was averaged somewhere
        plain = cgfd.media_volume(x, y, z, vx, vy, vz, vp, vs, rho, 100.0, 0.1, (1, 1, 1))
        assert np.abs(got[0] - plain[0]).max() > 1.0


def test_fluid_layer_keeps_zero_shear():
    x, y, z, ni, nj, nk = _grid()
    vx, vy, vz = _axes(x, y, z)
    X, Y, Z = np.meshgrid(vx, vy, vz, indexing="ij")
    vp = np.where(Z > -600.0, 1500.0, 4000.0).astype(np.float32)
    vs = np.where(Z > -600.0, 0.0, 2300.0).astype(np.float32)
    rho = np.where(Z > -600.0, 1000.0, 2500.0).astype(np.float32)
    got = cgfd.media_volume(x, y, z, vx, vy, vz, vp, vs, rho, 100.0, 0.1, (2, 2, 2))
    ref = MO.media_volume(x, y, z, ni, nj, nk, vx, vy, vz, vp, vs, rho, 100.0, 0.1, (2, 2, 2))
    for gq, rq in zip(got, ref):
        assert np.abs(gq - rq).max() <= 1e-6 * np.abs(rq).max()
    assert (got[1][3:-3, 3:-3, 3:-3] == 0).any()


def test_ghost_fill_and_checks():
    x, y, z, ni, nj, nk = _grid()
    vx, vy, vz = _axes(x, y, z)
    X, Y, Z = np.meshgrid(vx, vy, vz, indexing="ij")
    vp = (4000.0 - 0.3 * Z + 0.2 * X).astype(np.float32)
    a, _, _ = cgfd.media_volume(x, y, z, vx, vy, vz, vp, vp / 2, vp / 2)
    assert np.array_equal(a[0], a[3]) and np.array_equal(a[-1], a[-4])   # x: nearest
    assert np.array_equal(a[:, 0], a[:, 6]) and np.array_equal(a[:, -1], a[:, -4])  # y
    assert np.array_equal(a[:, :, 1], a[:, :, 5]) and np.array_equal(a[:, :, -2], a[:, :, -4])
    with pytest.raises(cgfd.CgfdError, match="increase"):
        cgfd.media_volume(x, y, z, vx[::-1].copy(), vy, vz, vp, vp, vp)
