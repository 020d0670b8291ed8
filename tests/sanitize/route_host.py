"""pytest plugin (loaded with -p route_host by tests/test_host_sanitizers.py):
the binding's host-side entry points -- those the sanitizer-instrumented
library named by CGFD_HOST_SANITIZED_LIB exports -- are called there, every
other one in the solver library."""
import ctypes as C
import os
import re
import subprocess


def pytest_configure(config):
    import cgfd
    path = os.environ["CGFD_HOST_SANITIZED_LIB"]
    lib = C.CDLL(path)
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True,
                         text=True, check=True).stdout
    names = set(re.findall(r"\bT\s+(cgfd_\w+)", out))
    real = cgfd._lib

    class Routed:
        def __getattr__(self, name):
            f = getattr(real, name)
            if name in names:
                g = getattr(lib, name)
                g.argtypes, g.restype = f.argtypes, f.restype
                f = g
            setattr(self, name, f)
            return f

    cgfd._lib = Routed()
