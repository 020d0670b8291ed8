"""CPU restatement of the reference's volume-media path (media_type =
volume): TEST INFRASTRUCTURE, only tests import it.

Follows src/mediaparas.cpp: read_volume_new (1273-1424: the sub-volume that
brackets the valid nodes), readdata (2140-2220), volume_discrete (376-440:
trilinear between bracketing samples via mathfunc::LocValue1d /
interp3d, src/mathfunc.cpp:294-328, 395-447), get2in1 / set_vel3d (872-923),
ApplySmooth / OverLimits (1712-1835: sub-cell samples where Vp jumps,
TwoinOne / average 838-914: density arithmetic, lambda and mu harmonic),
MediaStatistics (1837-1900: back to Vp, Vs, rho on valid nodes) and
common::equivalence_extend (src/common.cpp:136-166).  Plain Python over
small grids; float64 throughout (the reference's TypeDouble build).

Parity unpinned against the reference itself: mediaparas.cpp does not
compile with this image's g++ (TwoinOne compares its int* argument with 0,
an error in every language mode), so its outputs cannot be generated here;
the restatement is checked against exact cases (a volume linear in x, y, z
is reproduced exactly) and against the product, written independently.
"""
import numpy as np


def locate(v, a):
    """(L, R, value) as LocValue1d: bracketing indices on an increasing
    axis, the value clamped to its ends."""
    n = len(a)
    if v <= a[0]:
        return 0, 1, a[0]
    if v >= a[n - 1]:
        return n - 2, n - 1, a[n - 1]
    lo, hi = 0, n - 1
    while hi - lo > 1:
        m = (hi - lo) // 2 + lo
        if a[m] == v:
            return m, m + 1, v
        if a[m] > v:
            hi = m
        else:
            lo = m
    return lo, hi, v


def weights(X, x0):
    out = []
    for i in range(len(X)):
        w = 1.0
        for j in range(len(X)):
            if j != i:
                w *= (X[j] - x0) / (X[j] - X[i])
        out.append(w)
    return out


class Volume:
    def __init__(self, ax, fields, lo, hi):
        self.ax = [a[l:h + 1] for a, l, h in zip(ax, lo, hi)]
        self.f = [f[lo[0]:hi[0] + 1, lo[1]:hi[1] + 1, lo[2]:hi[2] + 1] for f in fields]

    def sample(self, p):
        ii, ww = [], []
        for d in range(3):
            L, _, q = locate(p[d], self.ax[d])
            ii.append(L)
            ww.append(weights(self.ax[d][L:L + 2], q))
        out = []
        for f in self.f:
            s = 0.0
            for a in range(2):
                for b in range(2):
                    for c in range(2):
                        s += ww[0][a] * ww[1][b] * ww[2][c] * float(f[ii[0] + a, ii[1] + b, ii[2] + c])
            out.append(s)
        return out  # vp, vs, rho


def media_volume(x, y, z, ni, nj, nk, vx, vy, vz, vp, vs, rho, crit_value, crit_perc,
                 samp=(1, 1, 1)):
    """(alpha, beta, rho) full arrays (ni+6, nj+6, nk+6) from a volume
    vp/vs/rho [nvx][nvy][nvz] on increasing axes vx, vy, vz."""
    c = [np.asarray(v, np.float64) for v in (x, y, z)]
    ax = [np.asarray(v, np.float64) for v in (vx, vy, vz)]
    V = slice(3, -3)
    lo, hi = [], []
    for d in range(3):
        val = c[d][V, V, V]
        lo.append(locate(val.min(), ax[d])[0])
        hi.append(locate(val.max(), ax[d])[1])
    vol = Volume(ax, [np.asarray(f, np.float64) for f in (vp, vs, rho)], lo, hi)
    shape = c[0].shape
    lam, mu, den, vel = (np.zeros(shape) for _ in range(4))
    for i in range(shape[0]):
        for j in range(shape[1]):
            for k in range(shape[2]):
                p, s, d = vol.sample((c[0][i, j, k], c[1][i, j, k], c[2][i, j, k]))
                m = d * s * s
                mu[i, j, k] = (m + m) / 2.0
                lam[i, j, k] = ((p * p * d - 2.0 * m) * 2) / 2.0
                den[i, j, k] = (d + d) / 2.0
                vel[i, j, k] = p if (0.0 < crit_value and 0.0 < crit_perc) else p + 9000e3

    def over(a, b):
        return abs(a - b) >= crit_value or abs(a - b) / min(a, b) >= crit_perc

    if max(samp) > 1:
        vec3 = [0.0, 2.0, 4.0]
        nl, nm, nd = lam.copy(), mu.copy(), den.copy()
        for i in range(3, ni + 3):
            for j in range(3, nj + 3):
                for k in range(3, nk + 3):
                    v0 = vel[i, j, k]
                    sx = samp[0] if over(v0, vel[i - 1, j, k]) or over(v0, vel[i + 1, j, k]) else 1
                    sy = samp[1] if over(v0, vel[i, j - 1, k]) or over(v0, vel[i, j + 1, k]) else 1
                    sz = samp[2] if over(v0, vel[i, j, k - 1]) or over(v0, vel[i, j, k + 1]) else 1
                    if sx == sy == sz == 1:
                        continue
                    rs = ms = ls = 0.0
                    ns = 0
                    for mi in range(1, sx + 1):
                        for mj in range(1, sy + 1):
                            for mk in range(1, sz + 1):
                                w = [weights(vec3, 1.0 + 2.0 / s_ * (m_ - 1 + 0.5))
                                     for s_, m_ in ((sx, mi), (sy, mj), (sz, mk))]
                                pt = [0.0, 0.0, 0.0]
                                for a in range(3):
                                    for b in range(3):
                                        for cc in range(3):
                                            ww = w[0][a] * w[1][b] * w[2][cc]
                                            for d in range(3):
                                                pt[d] += ww * c[d][i - 1 + a, j - 1 + b, k - 1 + cc]
                                p, s, dc = vol.sample(pt)
                                m = dc * s * s
                                l_ = p * p * dc - 2.0 * m
                                rs += 0.5 * (dc + dc)
                                ms = 0.0 if m < 1e-20 else ms + 0.5 / m + 0.5 / m
                                ls += 0.5 / l_ + 0.5 / l_
                                ns += 1
                    nd[i, j, k] = rs / ns
                    nm[i, j, k] = ns / ms if ms > 0 else 0.0
                    nl[i, j, k] = ns / ls
        lam, mu, den = nl, nm, nd
    out = [np.zeros(shape) for _ in range(3)]
    out[0][V, V, V] = np.sqrt((lam + 2.0 * mu) / den)[V, V, V]
    out[1][V, V, V] = np.sqrt(mu / den)[V, V, V]
    out[2][V, V, V] = den[V, V, V]
    for v in out:  # equivalence_extend
        for s in range(1, 4):
            v[3 - s, :, :] = v[3, :, :]
            v[ni + 2 + s, :, :] = v[ni + 2, :, :]
        for s in range(1, 4):
            v[:, 3 - s, :] = v[:, 3 + s, :]
            v[:, nj + 2 + s, :] = v[:, nj + 2, :]
        for s in range(1, 4):
            v[:, :, 3 - s] = v[:, :, 3 + s]
            v[:, :, nk + 2 + s] = v[:, :, nk + 2]
    return out
