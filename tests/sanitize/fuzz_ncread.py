"""Damaged NetCDF classic files against the readers (cgfd_read_media_volume_nc,
cgfd_read_focal_nc) of a sanitizer-instrumented build of the host code.

    python fuzz_ncread.py LIB SEED ITERATIONS WORKDIR

Seeds: volume media files of both classic versions and a finite-fault file,
written by scipy.  Each iteration overwrites 1-6 random spots of a seed's
first 400 bytes (single bytes, or 4-byte words such as 0xffffffff,
0x7fffffff, 0, 0x80000000) or cuts the file short, then calls both readers:
the size query and, when the sizes it returns are small, the full read into
arrays of those sizes.  A memory error aborts the process (AddressSanitizer,
halt_on_error); otherwise it prints how many reads succeeded and how many
were refused."""
import ctypes as C
import os
import random
import sys

import numpy as np
from scipy.io import netcdf_file


def seeds(workdir):
    rng = np.random.default_rng(0)
    out = []
    for version in (1, 2):
        p = os.path.join(workdir, f"volume{version}.nc")
        with netcdf_file(p, "w", version=version) as f:
            for name, n in (("x", 5), ("y", 4), ("depth", 6)):
                f.createDimension(name, n)
                f.createVariable(name, "f8", (name,))[:] = np.sort(rng.uniform(0, 1e3, n))
            for k in ("Vp", "Vs", "rho"):
                f.createVariable(k, "f4", ("x", "y", "depth"))[:] = rng.uniform(1, 8, (5, 4, 6))
        out.append(open(p, "rb").read())
    p = os.path.join(workdir, "focal.nc")
    with netcdf_file(p, "w") as f:
        f.createDimension("NP", 3)
        f.createDimension("NT", 5)
        f.DT = 0.01
        for k in ("Mxx", "Myy", "Mzz", "Mxy", "Mxz", "Myz"):
            f.createVariable(k, "f4", ("NP", "NT"))[:] = rng.uniform(-1, 1, (3, 5))
        for k in ("posx", "posy", "posz"):
            f.createVariable(k, "f8", ("NP",))[:] = np.arange(3.0)
    out.append(open(p, "rb").read())
    return out


def main(lib_path, seed, iterations, workdir):
    lib = C.CDLL(lib_path)
    corpus = seeds(workdir)
    rng = random.Random(seed)
    path = os.path.join(workdir, "damaged.nc").encode()
    ok = refused = 0
    vp = C.c_void_p
    for _ in range(iterations):
        b = bytearray(rng.choice(corpus))
        for _ in range(rng.randint(1, 6)):
            hdr = min(len(b), 400)
            if hdr < 8:
                break
            r = rng.random()
            if r < 0.5:
                b[rng.randrange(hdr)] = rng.randrange(256)
            elif r < 0.85:
                i = rng.randrange(hdr - 4)
                b[i:i + 4] = rng.choice([b"\xff\xff\xff\xff", b"\x7f\xff\xff\xff", b"\0\0\0\0",
                                         b"\x80\0\0\0", rng.randbytes(4)])
            else:
                del b[rng.randrange(len(b)):]
        with open(path, "wb") as f:
            f.write(bytes(b))
        n = [C.c_int(0) for _ in range(3)]
        st = lib.cgfd_read_media_volume_nc(path, *[C.byref(x) for x in n], *[None] * 6)
        if st == 0:
            sz = [x.value for x in n]
            if sz[0] * sz[1] * sz[2] <= 4_000_000 and max(sz) <= 1_000_000:
                arrs = [np.zeros(k) for k in sz] + [np.zeros(sz[0] * sz[1] * sz[2], np.float32)
                                                     for _ in range(3)]
                st = lib.cgfd_read_media_volume_nc(path, *[C.byref(x) for x in n],
                                                   *[vp(a.ctypes.data) for a in arrs])
        ok, refused = (ok + 1, refused) if st == 0 else (ok, refused + 1)
        npt, nt, dt = C.c_int(), C.c_int(), C.c_double()
        st = lib.cgfd_read_focal_nc(path, C.byref(npt), C.byref(nt), C.byref(dt), *[None] * 4)
        if st == 0 and npt.value * nt.value <= 4_000_000:
            arrs = [np.zeros(npt.value) for _ in range(3)] + \
                   [np.zeros(6 * npt.value * nt.value, np.float32)]
            st = lib.cgfd_read_focal_nc(path, C.byref(npt), C.byref(nt), C.byref(dt),
                                        *[vp(a.ctypes.data) for a in arrs])
        ok, refused = (ok + 1, refused) if st == 0 else (ok, refused + 1)
    print(f"reads ok {ok} refused {refused}")


if __name__ == "__main__":
    main(sys.argv[1], int(sys.argv[2]), int(sys.argv[3]), sys.argv[4])
