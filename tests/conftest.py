import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tti-fdmodeling_b200"), os.path.join(ROOT, "oracle"), os.path.dirname(__file__)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle_lib():
    import pyoracle

    pyoracle.load()
    return pyoracle


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library; builds it in-tree if it is missing (the host has nvcc)."""
    import ttifd

    if not os.path.exists(ttifd.LIB_PATH):
        import subprocess

        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tti-fdmodeling_b200"), "lib"], check=True)
    return ttifd.load()


@pytest.fixture(scope="session")
def gpu_free_lib(gpu_lib):
    """The same library, for its host-only entry points (no device is touched)."""
    return gpu_lib
