"""cgfd_count_nonfinite_noalloc, the allocation-free NaN/Inf count.

It exists for callers that cannot call cudaMalloc when they check a
wavefield (their memory pool owns the device, or they run where the
allocator's synchronisation is not allowed).  Its counts must equal those of
the existing entry point, cgfd_check_finite, which runs the same kernels on
scratch the solver allocated at create.  The file is named so that pytest
collects it last; it needs nothing from the other tests.
"""
import numpy as np
import pytest

import cgfd
import models

pytestmark = pytest.mark.gpu


def _fields_with_bad_values(m, rng, n_bad_per_comp):
    """Finite random wavefield (valid cells) with NaN / +Inf / -Inf planted
    at random valid cells; ghost cells stay zero."""
    out = np.zeros((9,) + m.shape, np.float32)
    for c in range(9):
        v = rng.standard_normal(m.shape).astype(np.float32)
        f = np.zeros(m.shape, np.float32)
        f[3:-3, 3:-3, 3:-3] = v[3:-3, 3:-3, 3:-3]
        k = n_bad_per_comp[c]
        if k:
            idx = rng.choice(m.ni * m.nj * m.nk, size=k, replace=False)
            ii, jj, kk = np.unravel_index(idx, (m.ni, m.nj, m.nk))
            bad = np.array([np.nan, np.inf, -np.inf], np.float32)[np.arange(k) % 3]
            f[ii + 3, jj + 3, kk + 3] = bad
        out[c] = f
    return out


def test_noalloc_count_matches_check_finite_on_two_calls_in_a_row():
    import torch
    m = models.small_flat(nt=4)
    s = cgfd.Solver(m.desc())
    m.load(s)
    rng = np.random.default_rng(2024)
    plans = [[3, 0, 5, 0, 0, 7, 1, 0, 2], [0, 1, 0, 0, 4, 0, 0, 0, 0]]
    stream = torch.cuda.current_stream().cuda_stream
    for plan in plans:  # two calls in a row on the shared scratch
        fields = _fields_with_bad_values(m, rng, plan)
        for c in range(9):
            s.set_field(c, fields[c])
        expect = s.check_finite()  # existing entry point
        dev = torch.from_numpy(fields).cuda()
        torch.cuda.synchronize()
        got = cgfd.count_nonfinite_noalloc(dev.data_ptr(), dev.numel(), stream)
        assert expect == sum(plan)
        assert got == expect
    s.close()


def test_noalloc_count_is_zero_for_finite_data_and_rejects_oversize():
    import torch
    x = torch.ones(1 << 20, device="cuda", dtype=torch.float32)
    assert cgfd.count_nonfinite_noalloc(x.data_ptr(), x.numel()) == 0
    with pytest.raises(cgfd.CgfdError) as e:
        # rejected on the host before any device access
        cgfd.count_nonfinite_noalloc(x.data_ptr(), cgfd.NOALLOC_MAX_VALUES + 1)
    assert e.value.status == cgfd.ERR_ARG
    assert "exceed" in str(e.value)
