"""pytest plugin (loaded with -p route_host_program by
tests/test_host_sanitizers.py): the host program tests run the
sanitizer-instrumented build named by CGFD_HOST_SANITIZED_PROGRAM."""
import os


def pytest_configure(config):
    import hostio
    hostio.HOST = os.environ["CGFD_HOST_SANITIZED_PROGRAM"]
