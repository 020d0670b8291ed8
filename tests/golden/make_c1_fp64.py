"""Generates tests/golden/c1_fp64_seismograms.npz: the FP64 CPU oracle's
(oracle/cgfd_oracle.cpp) surface seismograms of the 160x160x80 flat
half-space (models.config_c1: explosive Ricker source at 2 km, 12-cell
CFS-PML, dt 8 ms, 500 RK4 steps, 25 receivers), the reference against which
the GPU tests state the error of 16-bit field storage.  The oracle is pinned
on the reference's own runtime by tests/test_oracle_golden.py.  The model's
pre-processing (metric, CFS-PML profiles, wavelet) is the oracle's FP64
restatement, so no GPU and no solver library is needed; it takes a few
minutes on 8 cores:

    python tests/golden/make_c1_fp64.py [output file]
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "copara-cgfd3d_b200", "python"), os.path.join(ROOT, "oracle")):
    sys.path.insert(0, p)

import numpy as np  # noqa: E402

import models  # noqa: E402
import pyoracle  # noqa: E402


def main(out):
    models.use_preprocessing("oracle")
    m = models.config_c1()
    o = pyoracle.OracleSolver(m.desc(), 0)
    m.load(o)
    o.step(m.nt)
    seis = o.seismograms()[:3].astype(np.float64)
    np.savez_compressed(out, seis=seis, nsteps=m.nt, rcv=m.rcv_loc)
    print(out, seis.shape)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "c1_fp64_seismograms.npz"))
