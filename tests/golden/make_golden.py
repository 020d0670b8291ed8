"""Generates the golden vectors in tests/golden/ by running the reference's
own device runtime (oracle/_ref/ref_wavesim, built from the reference's
src/calculate.cu by oracle/ref/Makefile) on the parity cases of
tests/cases.py.  Needs a GPU; run as

    python tests/golden/make_golden.py [output dir [case ...]]

(default: tests/golden/ itself, every case).  Cases whose model spreads its
sources (SrcSmooth) run on oracle/_ref/ref_wavesim_smooth.  Each file holds the reference's
seismograms (full steps) and the stage output W on the valid cells (partial
steps), plus the digest of the inputs it was made from.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "copara-cgfd3d_b200", "python"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)

import numpy as np  # noqa: E402

import cases  # noqa: E402
import refio  # noqa: E402


def main(out_dir, names=None):
    os.makedirs(out_dir, exist_ok=True)
    for name in names or cases.CASES:
        m, nsteps, nstages, init = cases.build(name)
        r = refio.run(m, nsteps, init, nstages)
        payload = dict(digest=np.array(cases.model_digest(m, init)), nsteps=nsteps,
                       nstages=nstages, ref_secs=r["secs"])
        if nsteps:
            payload["seis"] = r["seis"]
        if nstages:
            payload["w"] = r["w"][:, 3:-3, 3:-3, 3:-3]
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **payload)
        print(name, "done", f"{r['secs']:.3f}s")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden"),
         sys.argv[2:])
