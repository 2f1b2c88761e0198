"""Shared test setup.

Markers: ``gpu`` -- needs a CUDA device and the built CUDA library.

The CPU oracle (oracle/libmfd_oracle.so) is the parity checker; it is built here from
oracle/mfd_oracle.cpp when missing.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

ORACLE_SO = os.path.join(ROOT, "oracle", "libmfd_oracle.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built CUDA library")


def _build_oracle():
    src = os.path.join(ROOT, "oracle", "mfd_oracle.cpp")
    if (not os.path.exists(ORACLE_SO)) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])


@pytest.fixture(scope="session")
def oracle_lib():
    from maxwellfdtd_b200 import _abi
    _build_oracle()
    return _abi.Library(ORACLE_SO, "oracle_")


@pytest.fixture(scope="session")
def oracle64(oracle_lib):
    import maxwellfdtd_b200 as M
    return M.B200(np.float64, library=oracle_lib)


@pytest.fixture(scope="session")
def oracle32(oracle_lib):
    import maxwellfdtd_b200 as M
    return M.B200(np.float32, library=oracle_lib)


@pytest.fixture(scope="session")
def gpu_lib():
    import maxwellfdtd_b200 as M
    return M.load_library()


def isapprox(a, b, rtol):
    """Julia ``isapprox(a, b; rtol)`` for arrays: norm(a-b) <= rtol*max(norm(a), norm(b))."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) <= rtol * max(np.linalg.norm(a), np.linalg.norm(b))


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = max(np.linalg.norm(a), np.linalg.norm(b))
    return 0.0 if den == 0 else float(np.linalg.norm(a - b) / den)
