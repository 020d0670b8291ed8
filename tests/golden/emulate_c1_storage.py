"""Seismogram error of emulated 16-bit field storage on the 160x160x80 flat
half-space (models.config_c1, 500 RK4 steps) against the FP64 oracle's
seismograms in c1_fp64_seismograms.npz: the FP64 oracle
(oracle/cgfd_oracle.cpp) rounds the stored field sets after every write as
orc_set_storage_emulation describes.  Each case takes about 8 minutes on 8
cores; without arguments it runs the cases the design notes quote:

    python tests/golden/emulate_c1_storage.py [case ...]
"""
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "copara-cgfd3d_b200", "python"), os.path.join(ROOT, "oracle")):
    sys.path.insert(0, p)

import numpy as np  # noqa: E402

import models  # noqa: E402
import pyoracle  # noqa: E402

FP16 = dict(ebits=5, mbits=10, adapt=12)
CASES = {
    "fp16_tw_difference": dict(flags=1, **FP16),
    "fp16_tw_difference_feedback": dict(flags=5, **FP16),
    "bfp8x14_tw_difference": dict(ebits=108, mbits=14, flags=1),
    "bfp8x14_tw_difference_feedback": dict(ebits=108, mbits=14, flags=5),
}


QUOTED = ["fp16_tw_difference_feedback", "bfp8x14_tw_difference",
          "bfp8x14_tw_difference_feedback"]


def main(names):
    models.use_preprocessing("oracle")
    gold = np.load(os.path.join(HERE, "c1_fp64_seismograms.npz"))["seis"]
    m = models.config_c1()
    for name in names:
        t = time.time()
        o = pyoracle.OracleSolver(m.desc(), 0)
        m.load(o)
        o.set_storage_emulation(**CASES[name])
        o.step(m.nt)
        u = o.seismograms()[:3].astype(np.float64)
        o.close()
        e = np.linalg.norm(u - gold) / np.linalg.norm(gold)
        pk = abs(np.abs(u).max() - np.abs(gold).max()) / np.abs(gold).max()
        print(f"{name:34s} rel-L2 {e:.3e}  peak {pk:.2e}  ({time.time() - t:.0f} s)", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or QUOTED)
