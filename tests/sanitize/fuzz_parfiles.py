"""Damaged par files against a sanitizer-instrumented build of the host
program in its --dump mode (reading and pre-processing, no GPU).

    python fuzz_parfiles.py PROGRAM PARFILES_DIR SEED ITERATIONS WORKDIR

Each iteration copies the committed par-file set and makes 1-4 edits to
SeisFD3D.conf, absorb.dat, source.dat, station.dat or the vmap file (a token
replaced by an odd value -- negative, zero, huge, nan, inf, empty, text --
or a line deleted, doubled or cut short), leaving the grid's dimensions
alone so that the pre-processing stays small.  The program must exit 0 or
with its own message (status 1); a sanitizer report or any other status
fails the run."""
import os
import random
import shutil
import subprocess
import sys

FILES = ["SeisFD3D.conf", "absorb.dat", "source.dat", "station.dat", "grid_vmap.dat"]
KEEP = ("ni ", "nj ", "nk ", "ni=", "nj=", "nk=", "vmap_dims", "vmap_gridpoints", "nt ",
        "full_wave", "sampling")
VALUES = ["-1", "0", "1", "2", "3", "7", "-7", "1000000", "2147483647", "-2147483648", "1e308",
          "nan", "inf", "", "abc", "9e+06", "0.5", "-0.0", "99", "40", "48", "33", "31", "32"]


def main(prog, parfiles, seed, iterations, work):
    rng = random.Random(seed)
    bad = []
    for it in range(iterations):
        d = os.path.join(work, "run")
        shutil.rmtree(d, ignore_errors=True)
        shutil.copytree(parfiles, d)
        for _ in range(rng.randint(1, 4)):
            p = os.path.join(d, rng.choice(FILES))
            lines = open(p).read().split("\n")
            i = rng.randrange(min(len(lines), 60))
            if any(lines[i].strip().startswith(k) for k in KEEP):
                continue
            r = rng.random()
            toks = lines[i].split(" ")
            if r < 0.6:
                toks[rng.randrange(len(toks))] = rng.choice(VALUES)
                lines[i] = " ".join(toks)
            elif r < 0.75:
                del lines[i]
            elif r < 0.85:
                lines.insert(i, lines[i])
            else:
                lines[i] = lines[i][:rng.randrange(len(lines[i]) + 1)]
            with open(p, "w") as f:
                f.write("\n".join(lines))
        pr = subprocess.run([prog, "SeisFD3D.conf", "--dump", "m.bin"], cwd=d,
                            capture_output=True, text=True, timeout=120)
        if pr.returncode not in (0, 1) or "Sanitizer" in pr.stderr or "runtime error" in pr.stderr:
            bad.append((it, pr.returncode, pr.stderr[-2000:]))
    for b in bad:
        print("FAILED", *b)
    print(f"runs {iterations} failed {len(bad)}")
    return 1 if bad else 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1], sys.argv[2], int(sys.argv[3]), int(sys.argv[4]), sys.argv[5]))
