"""Training and evaluation of the learned thin absorbing layer (the solver's
boundary MLP, cgfd_set_boundary_mlp), and the reflected-energy measure.

Setup: a flat half-space (free surface on top, absorbing layers on the other
five faces) whose interior region of I cells is surrounded by an absorbing
layer of w cells; the reference ("big") run is the same medium padded by P
cells on the absorbing faces (plus a 20-cell CFS-PML), so that nothing
reflected at its boundary reaches the interior region within the window.

Training (teacher forcing, one step at a time): the thin-layer solver (w = 4
cells of CFS-PML) is set to the big run's state on the thin domain and
stepped once; the target of each layer cell is the big run's state after
that step minus the thin solver's, in the MLP's normalised units (divided by
the cell's feature scale, stresses also by rho*vp).  The MLP is fitted to
these one-step residuals by Adam on gradients from the device kernel
(cgfd_mlp_gradient).  Then a gain per (depth in the layer, component) is
fitted by least squares weighted by the squared feature scale (the physical
size of the error), and all gains are multiplied by one relaxation factor
picked on a validation source by the reflected energy of whole runs: the
one-step fit is imperfect, and its errors compound over the steps.

Reflected-energy fraction (evaluation): sum over interior receivers and the
time window of (u_test - u_big)^2 over the sum of u_big^2, velocities only.
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np

import cgfd
import models

LFD = 3


@dataclasses.dataclass
class Setup:
    interior: tuple = (48, 48, 24)   # cells of the interior region (x, y, z)
    h: float = 100.0
    dt: float = 0.008
    vp: float = 6000.0
    vs: float = 3464.0
    rho: float = 2670.0
    pad: int = 60                    # big run: extra cells on each absorbing face
    steps: int = 200


def _flat(ni, nj, nk, s: Setup, nabs, nt, src, m6, f0):
    m = models.flat_halfspace(ni=ni, nj=nj, nk=nk, h=s.h, dt=s.dt, nt=nt, vp=s.vp, vs=s.vs,
                              rho=s.rho, nabs=nabs, n_side=1, src_depth=s.h, f0=f0,
                              t0=1.2 / f0, name="flat")
    nstf = 2 * (nt + 1)
    wave = cgfd.stf("Ricker", 0.0, 1.2 / f0, f0, nstf, s.dt / 2.0)[None, :].astype(np.float32)
    return dataclasses.replace(m, mnt_loc=np.array([src], np.int32),
                               mnt_m6=np.asarray(m6, np.float32)[None, :], mnt_stf=wave,
                               rcv_loc=np.zeros((0, 3), np.int32))


def domain(s: Setup, w: int, src_int, m6, f0, nt=None, big=False):
    """A model whose interior region (s.interior) is surrounded by w cells of
    CFS-PML on the absorbing faces (big: s.pad cells of medium plus a 20-cell
    PML); src_int: source (i, j, k) inside the interior region, k from the
    bottom.  Returns (model, offset of the interior region's first cell in
    the model's valid index space)."""
    I, J, K = s.interior
    if big:
        e = s.pad + 20
        nabs = (20, 20, 20, 20, 20, 0)
    else:
        e = w
        nabs = (w, w, w, w, w, 0)
    ni, nj, nk = I + 2 * e, J + 2 * e, K + e
    off = (e, e, e)
    src = (LFD + off[0] + src_int[0], LFD + off[1] + src_int[1], LFD + off[2] + src_int[2])
    return _flat(ni, nj, nk, s, nabs, nt or s.steps + 2, src, m6, f0), off


def interior_receivers(s: Setup, stride=6):
    """A grid of receivers in the interior region (interior indices)."""
    I, J, K = s.interior
    return np.array([(i, j, k) for i in range(2, I - 2, stride) for j in range(2, J - 2, stride)
                     for k in range(2, K - 2, stride)], np.int32)


def run_with_receivers(m, off, rcv_int, steps, mlp=None, width=4):
    loc = np.array([(LFD + off[0] + i, LFD + off[1] + j, LFD + off[2] + k) for i, j, k in rcv_int],
                   np.int32)
    m = dataclasses.replace(m, rcv_loc=loc)
    sol = cgfd.Solver(m.desc())
    m.load(sol)
    if mlp is not None:
        sol.set_boundary_mlp(width, mlp)
    sol.step(steps)
    seis = sol.seismograms()[:3, :, :steps]
    sol.close()
    return seis


def reflected_energy(u_test, u_big):
    return float(((u_test - u_big) ** 2).sum() / (u_big ** 2).sum())


def _full(arr_valid, ni, nj, nk):
    f = np.zeros((ni + 6, nj + 6, nk + 6), np.float32)
    f[LFD:LFD + ni, LFD:LFD + nj, LFD:LFD + nk] = arr_valid
    return f


def teacher_samples(s: Setup, src_int, m6, f0, width=4, per_step=2000, rng=None,
                    skip_quiet=1e-6):
    """Training samples of one source: features x of the thin solver's layer
    cells after one step from the big run's state, the normalised one-step
    residual t to the big run, each sample's feature scale and its depth in
    the layer (0 = the cell next to the domain's edge)."""
    rng = rng or np.random.default_rng(0)
    big, boff = domain(s, width, src_int, m6, f0, big=True)
    thin, toff = domain(s, width, src_int, m6, f0)
    sb = cgfd.Solver(big.desc())
    big.load(sb)
    st = cgfd.Solver(thin.desc())
    thin.load(st)
    zero = np.zeros(cgfd.MLP_PARAMS, np.float16)
    st.set_boundary_mlp(width, zero)  # layer cells and features; no correction
    cells = st.boundary_mlp_cells()
    ci = cells - LFD  # thin valid indices
    depth = np.minimum.reduce([ci[:, 0], thin.ni - 1 - ci[:, 0], ci[:, 1], thin.nj - 1 - ci[:, 1],
                               ci[:, 2]])
    # thin valid cell (0,0,0) sits at big valid index start
    start = (boff[0] - toff[0] + LFD, boff[1] - toff[1] + LFD, boff[2] - toff[2] + LFD)
    count = (thin.ni, thin.nj, thin.nk)
    xs, ts, ss, ds = [], [], [], []
    for n in range(s.steps):
        snap = sb.snapshot(start, count)  # big state on the thin domain, 9 comps
        for c in range(9):
            st.set_field(c, _full(snap[c], *count))
        st.step(1)
        sb.step(1)
        nxt = sb.snapshot(start, count)
        x, scale, z = st.boundary_mlp_features()
        keep = np.nonzero(scale > skip_quiet * max(scale.max(), 1e-30))[0]
        if len(keep) == 0:
            continue
        if len(keep) > per_step:
            keep = rng.choice(keep, per_step, replace=False)
        thin_now = np.stack([st.get_field(c)[LFD:-LFD, LFD:-LFD, LFD:-LFD] for c in range(9)])
        ii, jj, kk = ci[keep, 0], ci[keep, 1], ci[keep, 2]
        res = nxt[:, ii, jj, kk] - thin_now[:, ii, jj, kk]  # [9][m]
        norm = scale[keep][None, :] * np.where(np.arange(9)[:, None] < 3, 1.0, z[keep][None, :])
        xs.append(x[keep])
        ts.append((res / norm).T.astype(np.float32))
        ss.append(scale[keep])
        ds.append(depth[keep])
    sb.close()
    st.close()
    return np.concatenate(xs), np.concatenate(ts), np.concatenate(ss), np.concatenate(ds)


# parameter layout of the layer MLP (include/cgfd.h: CGFD_MLP_PARAMS)
NIN, NH, NOUT = 45, 64, 9


def init_weights(seed=0, scale=0.5):
    """Initial parameters: Xavier-scaled hidden layers, zero output layer (no
    correction to start from), as FP64."""
    rng = np.random.default_rng(seed)
    w = np.zeros(cgfd.MLP_PARAMS)
    w[:NH * NIN] = rng.standard_normal(NH * NIN) * scale / np.sqrt(NIN)
    o = NH * NIN + NH
    w[o:o + NH * NH] = rng.standard_normal(NH * NH) * scale / np.sqrt(NH)
    return w


def train(x, t, w0, iters=800, batch=20000, lr=1e-3, seed=0, log=None):
    """Adam on the device gradient, learning rate held and then decayed
    linearly over the last third; returns FP16 weights."""
    rng = np.random.default_rng(seed)
    w = w0.astype(np.float64)
    m = np.zeros_like(w)
    v = np.zeros_like(w)
    b1, b2, eps = 0.9, 0.999, 1e-8
    hist = []
    for it in range(1, iters + 1):
        idx = rng.choice(len(x), min(batch, len(x)), replace=False)
        loss, g = cgfd.mlp_gradient(w.astype(np.float16), x[idx], t[idx])
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        a = lr * min(1.0, 3.0 * (1.0 - it / iters) + 0.05)
        w -= a * (m / (1 - b1 ** it)) / (np.sqrt(v / (1 - b2 ** it)) + eps)
        hist.append(loss)
        if log and (it % 50 == 0 or it == 1):
            log(f"iter {it} loss {loss:.4e}")
    return w.astype(np.float16), hist


GAIN = 0.25  # the solver's output bound: corrections are GAIN*tanh(y/GAIN)


def _silu(a):
    return a / (1.0 + np.exp(-a))


def mlp_outputs(w, x, chunk=200000):
    """The bounded outputs GAIN*tanh(y/GAIN) of the layer MLP for features x
    (float64 on the host; used to fit the gains)."""
    w = np.asarray(w, np.float64)
    o1 = NH * NIN
    W1, b1 = w[:o1].reshape(NH, NIN), w[o1:o1 + NH]
    o2 = o1 + NH
    W2, b2 = w[o2:o2 + NH * NH].reshape(NH, NH), w[o2 + NH * NH:o2 + NH * NH + NH]
    o3 = o2 + NH * NH + NH
    W3, b3 = w[o3:o3 + NOUT * NH].reshape(NOUT, NH), w[o3 + NOUT * NH:]
    out = np.empty((len(x), NOUT))
    for q in range(0, len(x), chunk):
        a = np.asarray(x[q:q + chunk], np.float64)
        y = _silu(_silu(a @ W1.T + b1) @ W2.T + b2) @ W3.T + b3
        out[q:q + chunk] = GAIN * np.tanh(y / GAIN)
    return out


def fit_gains(w, x, t, scale, depth, width=4):
    """Per (depth, component) least-squares gain of the bounded output
    against the target, weighted by scale^2, clipped to [0, 1]: [width][9]."""
    y = mlp_outputs(w, x)
    g = np.zeros((width, NOUT))
    for d in range(width):
        m = depth == d
        if not m.any():
            continue
        s2 = (scale[m].astype(np.float64) ** 2)[:, None]
        num = (s2 * y[m] * t[m]).sum(0)
        den = (s2 * y[m] ** 2).sum(0)
        g[d] = np.clip(num / np.maximum(den, 1e-300), 0.0, 1.0)
    return g.astype(np.float32)


def run_layer(m, off, rcv, steps, mlp=None, gains=None, width=4):
    """Velocity seismograms of the interior receivers, with the learned
    correction (mlp, gains) if given."""
    loc = np.array([(LFD + off[0] + i, LFD + off[1] + j, LFD + off[2] + k) for i, j, k in rcv],
                   np.int32)
    m = dataclasses.replace(m, rcv_loc=loc)
    sol = cgfd.Solver(m.desc())
    m.load(sol)
    if mlp is not None:
        sol.set_boundary_mlp(width, mlp)
        if gains is not None:
            sol.set_boundary_mlp_gains(gains)
    sol.step(steps)
    seis = sol.seismograms()[:3, :, :steps]
    sol.close()
    return seis


def pick_relaxation(s: Setup, src_int, m6, f0, mlp, gains, factors=(0.1, 0.2, 0.35, 0.5, 0.75, 1.0)):
    """The factor on the gains with the least reflected energy over a whole
    run of one (validation) source; returns (factor, {factor: energy})."""
    rcv = interior_receivers(s)
    big, boff = domain(s, 4, src_int, m6, f0, big=True)
    u_big = run_with_receivers(big, boff, rcv, s.steps)
    m, off = domain(s, 4, src_int, m6, f0)
    res = {a: reflected_energy(run_layer(m, off, rcv, s.steps, mlp, gains * a), u_big)
           for a in factors}
    return min(res, key=res.get), res


def evaluate(s: Setup, src_int, m6, f0, mlp=None, gains=None, long_steps=0):
    """Reflected-energy fractions of the 20-cell PML, the 4-cell PML and the
    4-cell PML with the learned correction (if mlp is given) against the
    padded run over s.steps; with long_steps, also the 4-cell layers against
    the 20-cell PML over long_steps (no padded run is feasible that long)."""
    rcv = interior_receivers(s)
    big, boff = domain(s, 4, src_int, m6, f0, big=True)
    u_big = run_with_receivers(big, boff, rcv, s.steps)
    out = {}
    for name, w, net in (("pml20", 20, None), ("pml4", 4, None), ("pml4_mlp", 4, mlp)):
        if name == "pml4_mlp" and mlp is None:
            continue
        m, off = domain(s, w, src_int, m6, f0)
        out[name] = reflected_energy(run_layer(m, off, rcv, s.steps, net, gains), u_big)
    if long_steps:
        nt = long_steps + 2
        m20, o20 = domain(s, 20, src_int, m6, f0, nt=nt)
        u20 = run_layer(m20, o20, rcv, long_steps)
        m4, o4 = domain(s, 4, src_int, m6, f0, nt=nt)
        out[f"pml4_vs_pml20_{long_steps}"] = reflected_energy(run_layer(m4, o4, rcv, long_steps), u20)
        if mlp is not None:
            out[f"pml4_mlp_vs_pml20_{long_steps}"] = reflected_energy(
                run_layer(m4, o4, rcv, long_steps, mlp, gains), u20)
    return out


def main(n_train=12, iters=800, seed=7, long_steps=3000, out=None):
    """Trains on n_train random sources, picks the relaxation on a
    validation source and evaluates on a held-out one; prints a JSON line of
    the reflected-energy fractions; out: .npz for the weights and gains."""
    import json
    import sys
    s = Setup()
    rng = np.random.default_rng(seed)
    I, J, K = s.interior

    def draw():
        src = (int(rng.integers(8, I - 8)), int(rng.integers(8, J - 8)), int(rng.integers(4, K - 4)))
        return src, rng.standard_normal(6) * 1e16, float(rng.uniform(3.0, 6.0))

    t0 = time.time()
    parts = [teacher_samples(s, *draw(), rng=rng) for _ in range(n_train)]
    x, t, sc, dep = (np.concatenate([p[q] for p in parts]) for q in range(4))
    del parts
    t_data = time.time() - t0
    w, hist = train(x, t, init_weights(seed), iters=iters,
                    log=lambda m: print(m, file=sys.stderr))
    sub = rng.choice(len(x), min(len(x), 1000000), replace=False)
    gains = fit_gains(w, x[sub], t[sub], sc[sub], dep[sub])
    t_train = time.time() - t0 - t_data
    factor, tried = pick_relaxation(s, *draw(), w, gains)
    gains = gains * factor
    res = evaluate(s, *draw(), mlp=w, gains=gains, long_steps=long_steps)
    res.update(samples=int(len(x)), data_s=round(t_data, 1), train_s=round(t_train, 1),
               loss_first=hist[0], loss_last=hist[-1], target_ms=float((t ** 2).sum(1).mean()),
               relaxation=factor, relaxation_tried={str(k): v for k, v in tried.items()},
               gains=[[round(float(v), 4) for v in row] for row in gains])
    if out:
        np.savez(out, weights=w, gains=gains)
    print(json.dumps(res))
    return res


if __name__ == "__main__":
    import sys
    main(out=sys.argv[1] if len(sys.argv) > 1 else None)
