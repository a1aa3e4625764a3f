"""Shared pytest setup: the `gpu` marker, import paths for the package
(directory name is not an identifier) and the checkers in oracle/."""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "microgravity-cryogenic-multi-phase-sph-solver_b200")
ORACLE = os.path.join(REPO, "oracle")
TESTS = os.path.join(REPO, "tests")
for p in (PKG, ORACLE, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")
    config.addinivalue_line("markers", "slow: long-running check")


@pytest.fixture(scope="session")
def cuda_device():
    """Fails (does not skip) when the CUDA path cannot run: GPU tests must
    exercise the native library, never a fallback."""
    import cryo_cabi
    L = cryo_cabi.load()
    n = L.cryo_device_count()
    assert n > 0, "no CUDA device visible to libcryosph_b200.so"
    return 0
