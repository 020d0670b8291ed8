"""Generates the golden vectors in tests/golden/ by running the reference's
own device runtime (oracle/_ref/ref_wavesim, built from the reference's
src/calculate.cu by oracle/ref/Makefile) on the parity cases of
tests/cases.py.  Needs a GPU; run as

    python tests/golden/make_golden.py [output dir [case ...]]

(default: tests/golden/ itself, every case).  Cases whose model spreads its
sources (SrcSmooth) run on oracle/_ref/ref_wavesim_smooth.  Each file holds the reference's
seismograms (full steps) and the stage output W on the valid cells (partial
steps), plus the digest of the inputs it was made from.  The case
cases.OUTPUT_CASE also holds the reference's peak velocities and snapshot
samples of a run with a finite fault.
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


def outputs_case(out_dir):
    """The reference's focal source (C2DFocalPick / InterpFocus / LoadRmom),
    peak velocity (IterationFinalPV) and snapshots (C2DSnapPick / SWpick) in
    one run of cases.OUTPUT_CASE."""
    m = cases.build_outputs_case()
    pts = cases.snap_points()
    r = refio.run(m, m.nt, fields=False, focal=True, peak_velocity=True, snap_points=pts,
                  snap_tinv=cases.SNAP_TINV)
    np.savez_compressed(os.path.join(out_dir, f"{cases.OUTPUT_CASE}.npz"),
                        digest=np.array(cases.model_digest(m)), nsteps=m.nt,
                        ref_secs=r["secs"], seis=r["seis"], pv=r["pv"][:, 3:-3, 3:-3],
                        snap=r["snap"], snap_points=pts)
    print(cases.OUTPUT_CASE, "done", f"{r['secs']:.3f}s")


def main(out_dir, names=None):
    os.makedirs(out_dir, exist_ok=True)
    if not names or cases.OUTPUT_CASE in names:
        outputs_case(out_dir)
    for name in names or cases.CASES:
        if name == cases.OUTPUT_CASE:
            continue
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
