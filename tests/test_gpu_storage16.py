"""16-bit field storage (FP16 with per-component power-of-two scales, BF16):
the nine wavefields and the RK registers are stored at 16 bits, the
arithmetic stays FP32.  There is no reference counterpart to match bit for
bit; the checks are accuracy bounds against the FP64 oracle's seismograms
(tests/golden/c1_fp64_seismograms.npz, made by make_c1_fp64.py) and
against the solver's own FP32 storage (which matches the reference within
1e-5) on the same inputs, plus exact properties of the storage conversions
and scales.

Measured on a B200 (seismogram relative L2 of Vx..Vz), with the RK
accumulator stored as its difference from FW: small flat 60 steps FP16
1.10e-3 / BF16 8.9e-3 against FP32 storage; small hill FP16 1.39e-3 / BF16
2.9e-3; the 160x160x80 flat half-space, 500 steps, against the FP64 oracle:
FP16 3.7e-3, BF16 2.8e-2 (peak amplitude 0.23% / 0.03%).  (Storing tW
itself they were 1.7e-3 / 1.5e-2, 2.8e-3 / 9.3e-3 and 7.0e-3 / 6.3e-2.)
The bounds sit about 25% above the measurements: a regression shows.  Where
the FP16 error comes from (which stored set) is measured on the CPU in
test_storage_emulation.py.
"""
import os

import numpy as np
import pytest

import cgfd
import models
from helpers import rel_l2

pytestmark = pytest.mark.gpu

STORES = {"f16": cgfd.STORE_F16, "bf16": cgfd.STORE_BF16}


def _run(m, steps, storage):
    s = cgfd.Solver(m.desc(storage=storage))
    m.load(s)
    s.step(steps)
    seis, nbad, scales = s.seismograms(), s.check_finite(), s.field_scales()
    s.close()
    return seis, nbad, scales


@pytest.mark.parametrize("name,bound", [("small_flat", {"f16": 1.4e-3, "bf16": 1.1e-2}),
                                        ("small_hill", {"f16": 1.75e-3, "bf16": 3.6e-3})])
@pytest.mark.parametrize("store", list(STORES))
def test_16bit_storage_tracks_fp32_storage(name, bound, store):
    m = getattr(models, name)(nt=60)
    ref, nbad, _ = _run(m, 60, cgfd.STORE_F32)
    seis, nbad16, scales = _run(m, 60, STORES[store])
    assert nbad == 0 and nbad16 == 0
    e = rel_l2(seis[:3], ref[:3])
    assert e < bound[store], (name, store, e, scales)


@pytest.mark.parametrize("store,bound,peak", [("f16", 4.6e-3, 3e-3), ("bf16", 3.5e-2, 1e-3)])
def test_flat_halfspace_160x160x80_500_steps_16bit(store, bound, peak):
    """The FP16/BF16 variant of the 160x160x80 flat half-space model against
    the FP64 oracle's seismograms (and FP32 storage against the same, 1e-5)."""
    m = models.config_c1()
    gold = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                "c1_fp64_seismograms.npz"))["seis"]
    ref, _, _ = _run(m, m.nt, cgfd.STORE_F32)
    seis, nbad, scales = _run(m, m.nt, STORES[store])
    assert nbad == 0
    assert rel_l2(ref[:3], gold) < 1e-5, rel_l2(ref[:3], gold)
    e = rel_l2(seis[:3], gold)
    assert e < bound, (store, e)
    pk, pk_ref = np.abs(seis[:3]).max(), np.abs(gold).max()
    assert abs(pk - pk_ref) / pk_ref < peak, (store, e, abs(pk - pk_ref) / pk_ref)
    if store == "f16":
        assert scales[0] != 0 or scales[3] != 0  # the automatic scales were set
    else:
        assert scales == [0] * 9


@pytest.mark.parametrize("store,ulp", [("f16", 2.0 ** -11), ("bf16", 2.0 ** -8)])
def test_field_round_trip_and_rescale_are_exact(store, ulp):
    m = models.small_flat(nt=4)
    s = cgfd.Solver(m.desc(storage=STORES[store]))
    m.load(s)
    rng = np.random.default_rng(5)
    f = np.zeros(m.shape, np.float32)
    f[3:-3, 3:-3, 3:-3] = rng.standard_normal((m.ni, m.nj, m.nk)).astype(np.float32) * 100.0
    s.set_field(4, f)
    g = s.get_field(4)
    v = f[3:-3, 3:-3, 3:-3]
    assert np.all(np.abs(g[3:-3, 3:-3, 3:-3] - v) <= ulp * np.abs(v) + 1e-30)
    assert not np.any(g[:3]) and not np.any(g[-3:])  # ghosts stay zero
    # a power-of-two rescale does not change the values the fields stand for
    e = s.field_scales()
    e2 = [x + 3 for x in e]
    s.set_field_scales(e2)
    assert s.field_scales() == e2
    assert np.array_equal(s.get_field(4), g)
    s.close()


def test_accumulator_read_back_through_the_difference_form():
    """16-bit storage holds tW - FW; get_field / set_field of the tW set
    convert, so after single stages the accumulator a caller sees follows
    FP32 storage's within FP16 precision (measured <= 5.6e-4 per component
    after two stages), and a tW written by the caller reads back."""
    m = models.small_hill(nt=8)
    res = {}
    for k, st in (("f32", cgfd.STORE_F32), ("f16", cgfd.STORE_F16)):
        s = cgfd.Solver(m.desc(storage=st))
        m.load(s)
        s.step(3)
        s.rk_stage(0, 3, 1, 1, 1)
        s.rk_stage(1, 3, 1, 1, 1)
        res[k] = np.stack([s.get_field(c, cgfd.SET_TW) for c in range(9)])
        if k == "f16":
            t = res[k][4] * 0.5
            s.set_field(4, t, cgfd.SET_TW)
            back = s.get_field(4, cgfd.SET_TW)
            v = (slice(3, -3),) * 3
            assert rel_l2(back[v], t[v]) < 2e-3
        s.close()
    for c in range(9):
        assert rel_l2(res["f16"][c], res["f32"][c]) < 1.5e-3, (cgfd.COMPONENTS[c],)
