"""Shared test configuration.

Tests marked ``gpu`` need a B200 and the built native library; everything else
runs on CPU (oracle, host logic, library loading, gloo multi-process paths).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libhyowon_pm.so")


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.fixture(scope="session")
def oracle():
    from oracle.bindings import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def small_pm():
    return load_golden("small_pm.npz")


@pytest.fixture(scope="session")
def c1_kdk():
    return load_golden("c1_kdk.npz")


@pytest.fixture(scope="session")
def schedules():
    return load_golden("c1_schedule.npz")


@pytest.fixture(scope="session")
def c1_diag():
    return load_golden("c1_diag.npz")


@pytest.fixture(scope="session")
def pk_golden():
    return load_golden("pk.npz")


@pytest.fixture(scope="session")
def ic_golden():
    return load_golden("ic.npz")
