"""Shared test set-up: repository root on sys.path, the `gpu` marker, golden
fixture loading.  CPU tests (-m "not gpu") check the oracle against the
reference's golden fixtures and the host-side logic; GPU tests call the CUDA
library through its C ABI and compare with the oracle."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a library)")


def golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, name)) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def head_golden():
    return golden("head_L4_plummer1000.npz")


@pytest.fixture(scope="session")
def jacobi_golden():
    return golden("head_L3_jacobi.npz")


@pytest.fixture(scope="session")
def arrays_golden():
    return golden("arrays.npz")


@pytest.fixture(scope="session")
def stencil5_golden():
    return golden("head_L4_stencil5.npz")


@pytest.fixture(scope="session")
def cgsmooth_golden():
    return golden("head_L4_cgsmooth.npz")


@pytest.fixture(scope="session")
def cghead_golden():
    return golden("head_L4_cghead.npz")


@pytest.fixture(scope="session")
def periodic_golden():
    return golden("head_L4_periodic.npz")


@pytest.fixture(scope="session")
def periodic5_golden():
    return golden("head_L4_periodic5.npz")


@pytest.fixture(scope="session")
def outflow_golden():
    return golden("head_L4_outflow.npz")


@pytest.fixture(scope="session")
def timestep_golden():
    return golden("timestep_head_L4.npz")
