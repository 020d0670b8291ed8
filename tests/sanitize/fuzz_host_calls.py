"""Odd arguments against the host-side entry points of a sanitizer-
instrumented build of the host code: cgfd_metric_from_coords,
cgfd_cfs_factors, cgfd_stf, cgfd_angle2moment, cgfd_locate_points,
cgfd_source_smoothing and cgfd_media_volume on small grids whose coordinate
arrays carry a few odd values (0, -0, +-1e308, nan, +-inf, subnormals), with
odd scalars, layer widths, source nodes and volume axes -- always with
buffers of the sizes the header states.

    python fuzz_host_calls.py LIB SEED ITERATIONS

A memory error or undefined behaviour aborts the process; otherwise it
prints the count of each (entry point, status)."""
import ctypes as C
import random
import sys

import numpy as np


def main(lib_path, seed, iterations):
    lib = C.CDLL(lib_path)
    rng = random.Random(seed)
    nrng = np.random.default_rng(seed)

    def P(a):
        return C.c_void_p(a.ctypes.data)

    def odd():
        return rng.choice([0.0, -0.0, 1e308, -1e308, float("nan"), float("inf"), -float("inf"),
                           1e-310, rng.uniform(-1e4, 1e4)])

    def coords(ni, nj, nk, h=100.0):
        i, j, k = np.meshgrid(np.arange(ni + 6), np.arange(nj + 6), np.arange(nk + 6),
                              indexing="ij")
        x, y, z = (i * h).ravel(), (j * h).ravel(), ((k - (nk + 6)) * h).ravel()
        x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
        for a in (x, y, z):
            for _ in range(rng.randint(0, 3)):
                a[rng.randrange(a.size)] = odd()
        return x, y, z

    counts = {}
    for _ in range(iterations):
        ni, nj, nk = rng.randint(1, 9), rng.randint(1, 9), rng.randint(4, 9)
        x, y, z = coords(ni, nj, nk)
        N = x.size
        fn = rng.choice(["locate", "smooth", "media", "stf", "angle", "metric", "cfs"])
        if fn == "locate":
            n = rng.randint(0, 5)
            pos = nrng.uniform(-500, 1500, 3 * n)
            if n and rng.random() < 0.5:
                pos[rng.randrange(3 * n)] = odd()
            loc, posz = np.zeros(3 * n + 3, np.int32), np.zeros(n + 1)
            st = lib.cgfd_locate_points(ni, nj, nk, P(x), P(y), P(z),
                                        C.c_double(odd() if rng.random() < 0.3 else 9e6), n,
                                        P(pos), P(loc), P(posz))
        elif fn == "smooth":
            n = rng.randint(0, 4)
            loc = np.zeros(3 * n + 3, np.int32)
            pos = np.zeros(3 * n + 3)
            for q in range(n):
                if rng.random() < 0.9:
                    l3 = [rng.randint(3, ni + 2), rng.randint(3, nj + 2), rng.randint(3, nk + 2)]
                    g = (l3[0] * (nj + 6) + l3[1]) * (nk + 6) + l3[2]
                    pos[3 * q:3 * q + 3] = [x[g] + rng.uniform(-45, 45),
                                            y[g] + rng.uniform(-45, 45),
                                            z[g] + rng.uniform(-45, 45)]
                else:
                    l3 = [rng.randint(-2, 20) for _ in range(3)]
                    pos[3 * q:3 * q + 3] = nrng.uniform(-500, 1500, 3)
                loc[3 * q:3 * q + 3] = l3
            w = np.zeros(343 * n + 1)
            st = lib.cgfd_source_smoothing(ni, nj, nk, P(x), P(y), P(z),
                                           rng.choice([0, 1, 0, 1, -1, 2]), n, P(pos), P(loc),
                                           P(w))
        elif fn == "media":
            nv = [rng.randint(1, 5) for _ in range(3)]
            if rng.random() < 0.5:
                nv = [max(k, 2) for k in nv]
            ax = [np.sort(nrng.uniform(-2000, 3000, k)) for k in nv]
            for a in ax:
                if rng.random() < 0.2:
                    a[rng.randrange(a.size)] = odd()
            nvol = nv[0] * nv[1] * nv[2]
            vol = [nrng.uniform(0.5, 8, nvol).astype(np.float32) for _ in range(3)]
            for v in vol:
                if rng.random() < 0.3:
                    v[rng.randrange(v.size)] = np.float32(rng.choice([0.0, -1.0, 3e38, np.nan]))
            out = [np.zeros(N, np.float32) for _ in range(3)]
            samp = [rng.randint(1, 3) if rng.random() < 0.9 else rng.randint(-1, 4)
                    for _ in range(3)]
            st = lib.cgfd_media_volume(ni, nj, nk, P(x), P(y), P(z), *nv, *[P(a) for a in ax],
                                       *[P(v) for v in vol],
                                       C.c_double(odd() if rng.random() < 0.1 else 100.0),
                                       C.c_double(0.1), *samp, *[P(o) for o in out])
        elif fn == "stf":
            n = rng.randint(-2, 50)
            out = np.zeros(max(n, 0) + 1, np.float32)
            st = lib.cgfd_stf(rng.randint(-1, 8), C.c_double(odd()), C.c_double(odd()),
                              C.c_double(odd()), n, C.c_double(odd()), P(out))
        elif fn == "angle":
            m6 = np.zeros(6)
            st = lib.cgfd_angle2moment(C.c_double(odd()), C.c_double(odd()), C.c_double(odd()),
                                       P(m6))
        elif fn == "metric":
            outs = [np.zeros(N) for _ in range(10)]
            arr = (C.c_void_p * 10)(*[o.ctypes.data for o in outs])
            st = lib.cgfd_metric_from_coords(ni, nj, nk,
                                             C.c_double(odd() if rng.random() < 0.3 else 100.0),
                                             P(x), P(y), P(z), arr)
        else:
            dims = [ni, ni, nj, nj, nk, nk]
            nabs = np.array([rng.randint(0, dims[q]) if rng.random() < 0.9 else
                             rng.randint(-2, 12) for q in range(6)], np.int32)
            par = [np.array([odd() if rng.random() < 0.3 else 5000.0 for _ in range(6)])
                   for _ in range(3)]
            dl = [nrng.uniform(50, 150, k + 6) for k in (ni, nj, nk)]
            for a in dl:
                if rng.random() < 0.3:
                    a[rng.randrange(a.size)] = odd()
            outs = [np.zeros(k + 6) for _ in range(3) for k in (ni, nj, nk)]
            st = lib.cgfd_cfs_factors(ni, nj, nk, P(nabs), *[P(a) for a in par],
                                      *[P(a) for a in dl], *[P(o) for o in outs])
        counts[(fn, st)] = counts.get((fn, st), 0) + 1
    print("calls", sorted(counts.items()))


if __name__ == "__main__":
    main(sys.argv[1], int(sys.argv[2]), int(sys.argv[3]))
