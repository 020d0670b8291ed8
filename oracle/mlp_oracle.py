"""CPU restatement of the learned absorbing layer's MLP (test infrastructure:
only tests import it).

Forward: 45 -> 64 -> 64 -> 9 with SiLU after both hidden layers, parameters
(FP16 values, computed in float64 here) in the order W1 [64][45], b1 [64],
W2 [64][64], b2 [64], W3 [9][64], b3 [9]; loss = mean over samples of the
squared output error summed over the 9 outputs; gradients by
backpropagation.  The product's device kernels (csrc/mlp.cu) are checked
against these functions, and these against central finite differences.

Features of a layer cell (csrc/mlp.cu: features): the 9 components at the
cell and the next 4 cells along its inward normal, stresses over rho*vp,
divided by their largest magnitude (no correction below 1e-30); the applied
correction is correction() below, times the scale.
"""
import numpy as np

NIN, NH, NOUT = 45, 64, 9
OW1 = 0
OB1 = OW1 + NH * NIN
OW2 = OB1 + NH
OB2 = OW2 + NH * NH
OW3 = OB2 + NH
OB3 = OW3 + NOUT * NH
NPAR = OB3 + NOUT


def unpack(w):
    w = np.asarray(w, np.float64)
    return (w[OW1:OB1].reshape(NH, NIN), w[OB1:OW2], w[OW2:OB2].reshape(NH, NH), w[OB2:OW3],
            w[OW3:OB3].reshape(NOUT, NH), w[OB3:NPAR])


def silu(a):
    return a / (1.0 + np.exp(-a))


def dsilu(a):
    s = 1.0 / (1.0 + np.exp(-a))
    return s * (1.0 + a * (1.0 - s))


def forward(w, x):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    x = np.asarray(x, np.float64)
    a1 = x @ W1.T + b1
    a2 = silu(a1) @ W2.T + b2
    return silu(a2) @ W3.T + b3, a1, a2


GAIN = 0.25


def bounded(y):
    """The bounded output G*tanh(y/G)."""
    return GAIN * np.tanh(np.asarray(y, np.float64) / GAIN)


def correction(y, u, gains_of_cell):
    """The correction the solver applies to a cell in normalised units
    (csrc/mlp.cu: delta_kernel): d = gain * G*tanh(y/G), each component
    clamped so that u + d lies between 0 and u (u: the cell's own 9
    normalised values): the correction only damps."""
    d = np.asarray(gains_of_cell, np.float64) * bounded(y)
    u = np.asarray(u, np.float64)
    return np.clip(d, np.minimum(0.0, -u), np.maximum(0.0, -u))


def loss_grad(w, x, t):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    x = np.asarray(x, np.float64)
    y, a1, a2 = forward(w, x)
    n = len(x)
    e = y - np.asarray(t, np.float64)
    loss = float((e * e).sum() / n)
    dy = 2.0 * e / n
    g = np.zeros(NPAR)
    h2 = silu(a2)
    g[OW3:OB3] = (dy.T @ h2).reshape(-1)
    g[OB3:NPAR] = dy.sum(0)
    d2 = (dy @ W3) * dsilu(a2)
    h1 = silu(a1)
    g[OW2:OB2] = (d2.T @ h1).reshape(-1)
    g[OB2:OW3] = d2.sum(0)
    d1 = (d2 @ W2) * dsilu(a1)
    g[OW1:OB1] = (d1.T @ x).reshape(-1)
    g[OB1:OW2] = d1.sum(0)
    return loss, g


def init_weights(seed=0, scale=1.0):
    """Xavier-style initial parameters, rounded to FP16 values."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NPAR)
    w[OW1:OB1] = rng.standard_normal(NH * NIN) * scale / np.sqrt(NIN)
    w[OW2:OB2] = rng.standard_normal(NH * NH) * scale / np.sqrt(NH)
    w[OW3:OB3] = rng.standard_normal(NOUT * NH) * scale / np.sqrt(NH)
    return w.astype(np.float16)


def forward_fp16(w, x):
    """forward() with the device inference's roundings: the features and
    both hidden layers' SiLU outputs rounded to FP16 (the tensor-core
    operands), sums in float64."""
    W1, b1, W2, b2, W3, b3 = unpack(w)
    x = np.asarray(x, np.float32).astype(np.float16).astype(np.float64)
    h1 = silu(x @ W1.T + b1).astype(np.float16).astype(np.float64)
    h2 = silu(h1 @ W2.T + b2).astype(np.float16).astype(np.float64)
    return h2 @ W3.T + b3


def layer_cells(ni, nj, nk, nabs, width):
    """The layer cells of the solver's learned layer (csrc/solver.cu:
    cgfd_set_boundary_mlp), in its order (k, then j, then i: i fastest, as
    the solver's field layout): valid cells
    within `width` of an absorbing face (never the free surface), each with
    the inward unit step of its nearest face (ties x-, x+, y-, y+, z-) and
    its depth in the layer.  Returns (ijk (n, 3) in reference indices,
    step (n, 3), depth (n,))."""
    ijk, step, depth = [], [], []
    dirs = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1)]
    for k in range(nk):
        for j in range(nj):
            for i in range(ni):
                dist = [i if nabs[0] > 0 else 1 << 30, ni - 1 - i if nabs[1] > 0 else 1 << 30,
                        j if nabs[2] > 0 else 1 << 30, nj - 1 - j if nabs[3] > 0 else 1 << 30,
                        k if nabs[4] > 0 else 1 << 30]
                best, bd = -1, width
                for f in range(5):
                    if dist[f] < bd:
                        bd, best = dist[f], f
                if best < 0:
                    continue
                ijk.append((i + 3, j + 3, k + 3))
                step.append(dirs[best])
                depth.append(bd)
    return np.array(ijk), np.array(step), np.array(depth)


def apply_layer(fields, rho, vp, cells, w, gains, fp16=True):
    """The learned layer's correction of FW (fields [9][nx][ny][nz], float64,
    changed in place) after a step: features of every layer cell from the
    uncorrected fields, then all corrections added (csrc/mlp.cu)."""
    ijk, step, depth = cells
    n = len(ijk)
    z = np.array([rho[tuple(p)] * vp[tuple(p)] for p in ijk], np.float64)
    x = np.zeros((n, NIN))
    for s in range(5):
        p = ijk + s * step
        for c in range(NOUT):
            v = fields[c][p[:, 0], p[:, 1], p[:, 2]]
            x[:, s * NOUT + c] = v / z if c >= 3 else v
    scale = np.abs(x).max(axis=1)
    on = scale > 1e-30
    x[on] /= scale[on, None]
    y = forward_fp16(w, x) if fp16 else forward(w, x)[0]
    d = correction(y, x[:, :9], np.asarray(gains)[depth]) * scale[:, None]
    d[:, 3:] *= z[:, None]
    d[~on] = 0.0
    for c in range(NOUT):
        fields[c][ijk[:, 0], ijk[:, 1], ijk[:, 2]] += d[:, c]
    return fields
