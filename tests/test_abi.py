"""The C ABI: every entry point include/cgfd.h declares is exported by
libcgfd.so, argument errors come back as status codes (no GPU needed), and
the product library does not depend on the oracle."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cgfd.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^int\s+(cgfd_\w+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    names = declared()
    assert "cgfd_create" in names and "cgfd_step" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    import cgfd
    out = subprocess.run(["nm", "-D", "--defined-only", cgfd.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT\s+(cgfd_\w+)", out))
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing
    for n in declared():
        assert hasattr(cgfd._lib, n)


def test_binding_covers_every_declared_symbol():
    import cgfd
    assert sorted(cgfd.EXPORTED) == declared()


def test_every_entry_point_keeps_exceptions_inside():
    """Every definition of a declared entry point runs its body between
    CGFD_ABI_BEGIN and CGFD_ABI_END (csrc/abi_guard.h), so a host allocation
    or thread failure returns CGFD_ERR_NOMEM instead of unwinding into the
    caller; and every declared entry point is defined exactly once."""
    csrc = os.path.join(ROOT, "copara-cgfd3d_b200", "csrc")
    seen = {}
    for fn in sorted(os.listdir(csrc)):
        if not fn.endswith((".cu", ".cpp")):
            continue
        lines = open(os.path.join(csrc, fn)).read().split("\n")
        for i, line in enumerate(lines):
            m = re.match(r'^(?:extern "C" )?int (cgfd_\w+)\(', line)
            if not m:
                continue
            j = i
            while not lines[j].rstrip().endswith(("{", ";")):
                j += 1
            if lines[j].rstrip().endswith(";"):
                continue
            k = lines.index("}", j)
            seen[m.group(1)] = seen.get(m.group(1), 0) + 1
            assert lines[j + 1].strip() == "CGFD_ABI_BEGIN", (fn, m.group(1))
            assert lines[k - 1].strip().startswith("CGFD_ABI_END("), (fn, m.group(1))
    assert sorted(seen) == declared()
    assert all(v == 1 for v in seen.values())


def test_a_c99_host_builds_and_calls_the_library(tmp_path):
    """include/cgfd.h compiles as strict C99 (-pedantic, no warnings), a C
    program links libcgfd.so and calls it: a host-side entry point returns
    the reference's strike/dip/rake tensor, and cgfd_create refuses a zeroed
    description with CGFD_ERR_ARG and its text, without touching a GPU."""
    import shutil
    import cgfd
    if shutil.which("gcc") is None:
        pytest.skip("gcc needed")
    exe = str(tmp_path / "abi_c_caller")
    lib_dir = os.path.dirname(cgfd.LIB_PATH)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                        "-I" + os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "abi_c_caller.c"), "-L" + lib_dir, "-lcgfd",
                        "-Wl,-rpath," + lib_dir, "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, (out.stdout, out.stderr)
    f = out.stdout.split()
    assert f[0] == "abi" and f[2] == "m6"
    ref = cgfd.angle2moment(30.0, 60.0, 90.0)
    assert [float(v) for v in f[3:6]] == pytest.approx(list(ref[:3]), abs=1e-6)
    assert f[6] == "create" and int(f[7]) == cgfd.ERR_ARG and "bad grid" in out.stdout


def test_binding_refuses_arrays_of_the_wrong_size():
    """The C ABI reads exactly the model's number of values through each
    pointer; the binding checks the sizes first, so a short array is a
    ValueError, never a read past its end (no GPU: the checks come before
    any library call)."""
    import numpy as np
    import cgfd
    s = object.__new__(cgfd.Solver)
    s._h, s._owned, s.shape = None, False, (10, 9, 8)
    n = 10 * 9 * 8
    with pytest.raises(ValueError, match="metric array: 719 values, the model needs 720"):
        s.upload_metric(*[np.zeros(n)] * 3, np.zeros(n - 1))
    with pytest.raises(ValueError, match="media array"):
        s.upload_media(np.zeros(n), np.zeros((10, 9, 7)), np.zeros(n))
    prof = [np.zeros(k) for k in s.shape]
    with pytest.raises(ValueError, match="PML profile: 10 values, the model needs 9"):
        s.upload_pml(prof, (prof[0], prof[0], prof[2]), prof)
    with pytest.raises(ValueError, match="MLP weights"):
        s.set_boundary_mlp(4, np.zeros(cgfd.MLP_PARAMS - 1))
    with pytest.raises(ValueError, match="moment tensors: 12 values, the model needs 6"):
        s.upload_moments([[5, 5, 5]], np.zeros(12), np.zeros((1, 10)))
    with pytest.raises(ValueError, match="force vectors"):
        s.upload_forces([[5, 5, 5], [6, 6, 6]], np.zeros(3), np.zeros((2, 10)))
    s._mlp_width = 4
    with pytest.raises(ValueError, match="layer gains: 9 values, the model needs 36"):
        s.set_boundary_mlp_gains(np.ones(9))


def test_product_library_has_no_oracle_dependency():
    import cgfd
    out = subprocess.run(["nm", "-D", cgfd.LIB_PATH], capture_output=True, text=True).stdout
    assert "orc_" not in out
    ldd = subprocess.run(["ldd", cgfd.LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in ldd


@pytest.mark.parametrize("field,value", [
    ("ni", 0), ("nk", 2), ("steph", 0.0), ("stept", -1.0), ("hybrid_grid", 0),
    ("con_index", 2), ("con_index", 40), ("storage", 9), ("kernel", 7)])
def test_create_rejects_bad_descriptions(field, value):
    import cgfd
    d = cgfd.make_desc(20, 20, 20, 100.0, 0.005, 10, 10, (4, 4, 4, 4, 4, 0))
    setattr(d, field, value)
    with pytest.raises(cgfd.CgfdError) as e:
        cgfd.Solver(d)
    assert e.value.status == cgfd.ERR_ARG
    assert cgfd.last_error(None)


def test_create_rejects_pml_on_top_and_oversized_pml():
    import cgfd
    d = cgfd.make_desc(20, 20, 20, 100.0, 0.005, 10, 10, (4, 4, 4, 4, 4, 2))
    with pytest.raises(cgfd.CgfdError) as e:
        cgfd.Solver(d)
    assert e.value.status == cgfd.ERR_ARG and "free surface" in cgfd.last_error(None)
    d = cgfd.make_desc(20, 20, 20, 100.0, 0.005, 10, 10, (12, 12, 4, 4, 4, 0))
    with pytest.raises(cgfd.CgfdError):
        cgfd.Solver(d)
    # widths whose sum overflows an int, and a grid beyond 2^20 cells a side
    big = 2 ** 31 - 1
    d = cgfd.make_desc(20, 20, 20, 100.0, 0.005, 10, 10, (big, big, 4, 4, 4, 0))
    with pytest.raises(cgfd.CgfdError, match="PML wider than the grid"):
        cgfd.Solver(d)
    d = cgfd.make_desc(big - 6, 20, 20, 100.0, 0.005, 10, 10, (4, 4, 4, 4, 4, 0))
    with pytest.raises(cgfd.CgfdError, match="above 2\\^20"):
        cgfd.Solver(d)


@pytest.mark.parametrize("kernel", [1, 2])
def test_16bit_storage_needs_the_default_kernel(kernel):
    import cgfd
    d = cgfd.make_desc(20, 20, 20, 100.0, 0.005, 10, 10, (4, 4, 4, 4, 4, 0),
                       storage=cgfd.STORE_BF16, kernel=kernel)
    with pytest.raises(cgfd.CgfdError) as e:
        cgfd.Solver(d)
    assert e.value.status == cgfd.ERR_ARG
    assert "16-bit" in cgfd.last_error(None)


def test_noalloc_limit_is_the_header_limit():
    """cgfd_count_nonfinite_noalloc refuses more than CGFD_NOALLOC_MAX_VALUES
    values before touching the device, and takes the size itself: on a host
    pointer the limit passes the size check and fails the device-memory one
    (no GPU needed).  The binding's constant is the header's."""
    import ctypes as C

    import cgfd
    hdr = open(HEADER).read()
    lim = int(re.search(r"#define\s+CGFD_NOALLOC_MAX_VALUES\s+(\d+)", hdr).group(1))
    assert cgfd.NOALLOC_MAX_VALUES == lim
    host = (C.c_float * 4)()
    for n, text in ((lim + 1, "exceed the fixed scratch"), (lim, "not device memory")):
        out = C.c_longlong(-1)
        st = cgfd._lib.cgfd_count_nonfinite_noalloc(C.cast(host, C.c_void_p), n, C.byref(out),
                                                    None)
        assert st == cgfd.ERR_ARG and text in cgfd.last_error(None), (n, cgfd.last_error(None))


def test_handle_less_errors_are_per_thread():
    """The last error of a call without a handle is kept per host thread."""
    import threading

    import cgfd
    d = cgfd.make_desc(20, 20, 20, 100.0, 0.005, 10, 10, (4, 4, 4, 4, 4, 2))
    with pytest.raises(cgfd.CgfdError):
        cgfd.Solver(d)
    mine = cgfd.last_error(None)
    seen = []

    def other():
        seen.append(cgfd.last_error(None))
        bad = cgfd.make_desc(0, 20, 20, 100.0, 0.005, 10, 10, (4, 4, 4, 4, 4, 0))
        with pytest.raises(cgfd.CgfdError):
            cgfd.Solver(bad)
        seen.append(cgfd.last_error(None))

    t = threading.Thread(target=other)
    t.start()
    t.join()
    assert seen[0] == "" and seen[1] and seen[1] != mine
    assert cgfd.last_error(None) == mine
