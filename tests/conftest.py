"""Test configuration: markers and import paths.

`-m gpu` tests need a B200 and the built libraries (libcgfd.so, and the
reference parity driver oracle/_ref/ref_wavesim); `-m "not gpu"` tests run on
the CPU: the oracle against the reference's golden vectors, the host-side
pre-processing, and the C ABI's symbol table.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "copara-cgfd3d_b200", "python"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "tests"), os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libraries")
    config.addinivalue_line("markers", "slow: longer full-size parity runs")
