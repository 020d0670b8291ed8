"""The pure parts of bench.py on the CPU: the algorithmic bytes behind the
roofline, the workload names (and the thin-layer variants), the committed
traffic lookup and the config dict both arms print."""
import numpy as np

import models

# algorithmic bytes per step of the 600x600x250 hill, as its bench line reports them
ALG_600 = 69246720000


def _bench():
    import bench
    return bench


def test_algorithmic_bytes_of_a_flat_model():
    """144 state values per cell and step, 48 bytes of media coefficients
    per cell (3 per stage, FP32), 144 FP32 auxiliary values per (cell, PML
    direction) pair; a trivial metric costs nothing."""
    bench = _bench()
    m = models.small_flat(nt=4)
    pairs = ((m.nabs[0] + m.nabs[1]) * m.nj * m.nk + (m.nabs[2] + m.nabs[3]) * m.ni * m.nk +
             (m.nabs[4] + m.nabs[5]) * m.ni * m.nj)
    expect = 144 * 4 * m.cells + 144 * 4 * pairs + 3 * 4 * 4 * m.cells
    assert bench.algorithmic_bytes_per_step(m) == expect
    expect16 = 144 * 2 * m.cells + 144 * 4 * pairs + 3 * 4 * 4 * m.cells
    assert bench.algorithmic_bytes_per_step(m, elem=2) == expect16


def test_curved_metric_adds_its_coefficients():
    bench = _bench()
    m = models.small_hill(nt=4)
    flat_like = 3 * 4 * 4 * m.cells
    b = bench.algorithmic_bytes_per_step(m)
    pairs = ((m.nabs[0] + m.nabs[1]) * m.nj * m.nk + (m.nabs[2] + m.nabs[3]) * m.ni * m.nk +
             (m.nabs[4] + m.nabs[5]) * m.ni * m.nj)
    assert b - 144 * 4 * (m.cells + pairs) > flat_like


def test_workload_names_and_traffic_lookup():
    bench = _bench()
    assert bench.workload_name("hill600") == "gaussian_hill_600x600x250_random_layers_pml20"
    assert bench.workload_name("hill600", 4, True) == "gaussian_hill_600x600x250_random_layers_pml4_mlp"
    assert bench.workload_name("flat160", 6) == "flat_halfspace_160x160x80_pml6"
    t, shape = bench.committed_traffic(bench.workload_name("hill600"), "fused")
    assert t is not None and 1.0 < t / (ALG_600 / 4) < 1.2 and len(shape) == 3
    assert bench.committed_traffic("no_such_workload", "fused") == (None, None)


def test_config_dict_keys():
    bench = _bench()
    m = models.small_flat(nt=4)
    c = bench.config_dict("flat160", m)
    assert set(c) == {"workload", "cells", "grid", "pml_cells", "storage", "receivers", "l2"}
    assert c["cells"] == m.cells and c["grid"] == [m.ni, m.nj, m.nk]
    assert np.array_equal(c["pml_cells"], list(m.nabs))
