"""The CPU restatement of the learned layer's MLP: its gradient against
central finite differences (the oracle the device kernels are checked
against)."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "oracle"))
import mlp_oracle as M  # noqa: E402


def test_parameter_count_matches_the_abi():
    assert M.NPAR == 7689


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    w = M.init_weights(1).astype(np.float64)
    x = rng.uniform(-1, 1, (7, M.NIN))
    t = rng.standard_normal((7, M.NOUT)) * 0.1
    loss, g = M.loss_grad(w, x, t)
    idx = np.concatenate([rng.choice(np.arange(a, b), 6, replace=False) for a, b in
                          [(M.OW1, M.OB1), (M.OB1, M.OW2), (M.OW2, M.OB2), (M.OB2, M.OW3),
                           (M.OW3, M.OB3), (M.OB3, M.NPAR)]])
    eps = 1e-6
    for q in idx:
        wp, wm = w.copy(), w.copy()
        wp[q] += eps
        wm[q] -= eps
        fd = (M.loss_grad(wp, x, t)[0] - M.loss_grad(wm, x, t)[0]) / (2 * eps)
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(fd)), (q, fd, g[q])


def test_correction_only_damps():
    rng = np.random.default_rng(11)
    y = rng.standard_normal((5000, M.NOUT))
    u = rng.uniform(-1, 1, (5000, M.NOUT))
    g = rng.uniform(0, 2, (5000, M.NOUT))
    d = M.correction(y, u, g)
    raw = g * M.bounded(y)
    new = u + d
    # every component moves toward zero, never past it
    assert (np.abs(new) <= np.abs(u)).all() and (new * u >= 0).all()
    # corrections that already do so are kept as they are
    keep = (np.abs(u + raw) <= np.abs(u)) & ((u + raw) * u >= 0)
    assert keep.any() and (~keep).any()
    assert np.array_equal(d[keep], raw[keep])
