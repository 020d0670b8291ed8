"""The host-side code of the library -- the pre-processing (setup.cpp) and
the NetCDF reader and writer (ncread.cpp, ncinput.cpp, ncwrite.cpp) -- built
with AddressSanitizer and UndefinedBehaviorSanitizer on the CPU:

* the host pre-processing and reader tests (vmap grid, metric, CFS-PML,
  wavelets, point location and smoothing, volume media, NetCDF round trips
  and errors) run with the binding's host entry points routed to the
  instrumented build (tests/sanitize/route_host.py);
* the host program (wavesim_b200, host/wavesim.cpp, built the same way over
  the instrumented host code) runs its par-file tests;
* the host-side entry points take 2000 calls with odd arguments (nan, inf,
  huge and subnormal coordinates and scalars, layers wider than the grid,
  sources off the grid; tests/sanitize/fuzz_host_calls.py);
* the host program reads 120 damaged par-file sets in its --dump mode
  (tests/sanitize/fuzz_parfiles.py);
* the NetCDF readers take 1500 damaged files (random header bytes and words,
  files cut short; tests/sanitize/fuzz_ncread.py).

Any out-of-bounds access, use after free or undefined behaviour aborts the
child process, which fails the test."""
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.join(ROOT, "tests")
CSRC = os.path.join(ROOT, "copara-cgfd3d_b200", "csrc")
SOURCES = [os.path.join(CSRC, f) for f in ("setup.cpp", "ncread.cpp", "ncinput.cpp",
                                           "ncwrite.cpp")] + \
          [os.path.join(HERE, "sanitize", "host_stub.cpp")]
HOST_TESTS = ["test_setup.py", "test_grid_vmap.py", "test_source_locate.py",
              "test_media_volume.py", "test_ncread.py"]


def _libasan():
    if shutil.which("g++") is None:
        return None
    p = subprocess.run(["g++", "-print-file-name=libasan.so"], capture_output=True,
                       text=True).stdout.strip()
    return os.path.realpath(p) if os.path.isabs(p) and os.path.exists(p) else None


@pytest.fixture(scope="module")
def sanitized(tmp_path_factory):
    asan = _libasan()
    if asan is None:
        pytest.skip("g++ with AddressSanitizer is needed")
    lib = str(tmp_path_factory.mktemp("sanitized") / "libcgfd_host_sanitized.so")
    subprocess.run(["g++", "-shared", "-fPIC", "-g", "-O1", "-std=c++17", "-pthread",
                    "-fsanitize=address,undefined,float-cast-overflow",
                    "-fno-omit-frame-pointer", "-fno-sanitize-recover=all", *SOURCES,
                    "-o", lib], check=True)
    env = dict(os.environ, LD_PRELOAD=asan, UBSAN_OPTIONS="print_stacktrace=1",
               ASAN_OPTIONS="detect_leaks=0:halt_on_error=1",
               CGFD_HOST_SANITIZED_LIB=lib,
               PYTHONPATH=os.pathsep.join([os.path.join(HERE, "sanitize"),
                                           os.environ.get("PYTHONPATH", "")]))
    return lib, env


def test_host_preprocessing_under_sanitizers(sanitized):
    _, env = sanitized
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "route_host",
                        "-p", "no:cacheprovider", "-m", "not gpu",
                        *[os.path.join(HERE, t) for t in HOST_TESTS]],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, (r.stdout[-4000:], r.stderr[-4000:])
    assert " passed" in r.stdout


def test_netcdf_readers_on_damaged_files_under_sanitizers(sanitized, tmp_path):
    lib, env = sanitized
    r = subprocess.run([sys.executable, os.path.join(HERE, "sanitize", "fuzz_ncread.py"),
                        lib, "7", "1500", str(tmp_path)],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, (r.stdout[-4000:], r.stderr[-4000:])
    assert "reads ok" in r.stdout


@pytest.fixture(scope="module")
def sanitized_program(sanitized):
    lib, env = sanitized
    import cgfd
    d = os.path.dirname(lib)
    prog = os.path.join(d, "wavesim_sanitized")
    subprocess.run(["g++", "-g", "-O1", "-std=c++17", "-pthread",
                    "-fsanitize=address,undefined,float-cast-overflow",
                    "-fno-omit-frame-pointer", "-fno-sanitize-recover=all",
                    os.path.join(ROOT, "copara-cgfd3d_b200", "host", "wavesim.cpp"),
                    os.path.join(CSRC, "ncwrite.cpp"),
                    "-L" + d, "-lcgfd_host_sanitized",
                    "-L" + os.path.dirname(cgfd.LIB_PATH), "-lcgfd",
                    "-Wl,-rpath," + d, "-Wl,-rpath," + os.path.dirname(cgfd.LIB_PATH),
                    "-o", prog], check=True)
    env = dict(env, CGFD_HOST_SANITIZED_PROGRAM=prog)
    env.pop("LD_PRELOAD")  # the program links the sanitizer runtime itself
    return prog, env


def test_host_program_under_sanitizers(sanitized_program):
    _, env = sanitized_program
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "route_host_program",
                        "-p", "no:cacheprovider", "-m", "not gpu",
                        os.path.join(HERE, "test_host_parfiles.py")],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, (r.stdout[-4000:], r.stderr[-4000:])
    assert " passed" in r.stdout


def test_host_program_on_damaged_par_files_under_sanitizers(sanitized_program, tmp_path):
    prog, env = sanitized_program
    r = subprocess.run([sys.executable, os.path.join(HERE, "sanitize", "fuzz_parfiles.py"), prog,
                        os.path.join(HERE, "golden", "parfiles"), "11", "120", str(tmp_path)],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, (r.stdout[-4000:], r.stderr[-4000:])
    assert "failed 0" in r.stdout


def test_host_entry_points_on_odd_arguments_under_sanitizers(sanitized):
    lib, env = sanitized
    r = subprocess.run([sys.executable, os.path.join(HERE, "sanitize", "fuzz_host_calls.py"),
                        lib, "5", "2000"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, (r.stdout[-4000:], r.stderr[-4000:])
    assert "calls" in r.stdout
