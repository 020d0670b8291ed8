"""The host side of the learned layer's training (python/learned_layer.py)
on the CPU: the bounded MLP outputs the gains are fitted on agree with the
MLP oracle's forward pass, the gain fit recovers known gains (and clips them
to [0, 1]), and the initial parameters start from no correction."""
import numpy as np

import learned_layer as L
import mlp_oracle as M


def _weights(seed):
    rng = np.random.default_rng(seed)
    w = L.init_weights(seed)
    w[M.OW3:] = rng.standard_normal(M.NPAR - M.OW3) * 0.3
    return w


def test_bounded_outputs_match_the_oracle_forward_pass():
    w = _weights(1)
    x = np.random.default_rng(2).uniform(-1, 1, (500, M.NIN))
    y = M.forward(w, x)[0]
    np.testing.assert_allclose(L.mlp_outputs(w, x), M.bounded(y), rtol=1e-12, atol=1e-14)


def test_gain_fit_recovers_known_gains():
    w = _weights(3)
    rng = np.random.default_rng(4)
    n = 4000
    x = rng.uniform(-1, 1, (n, M.NIN))
    depth = rng.integers(0, 4, n)
    scale = rng.uniform(0.1, 2.0, n).astype(np.float32)
    true = rng.uniform(0.0, 1.0, (4, 9))
    true[2, 5] = 1.7  # above the clip
    true[3, 1] = -0.4  # below it
    y = L.mlp_outputs(w, x)
    t = y * true[depth]
    g = L.fit_gains(w, x, t, scale, depth, width=4)
    expect = np.clip(true, 0.0, 1.0)
    np.testing.assert_allclose(g, expect, rtol=1e-5, atol=1e-6)


def test_initial_parameters_give_no_correction():
    w = L.init_weights(0)
    assert w.size == M.NPAR and not w[M.OW3:].any()
    x = np.random.default_rng(5).uniform(-1, 1, (100, M.NIN))
    assert not L.mlp_outputs(w, x).any()
    assert L.reflected_energy(np.ones(4), np.ones(4)) == 0.0
