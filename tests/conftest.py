"""Shared fixtures: the package (imported by path, its directory name has a hyphen), the checker,
and GPU gating. GPU tests are marked ``gpu``; everything else runs on CPU."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
ORACLE_DIR = os.path.join(ROOT, "oracle")
if ORACLE_DIR not in sys.path:
    sys.path.insert(0, ORACLE_DIR)

PKG = "nuppn_modular2-ininet3_b200"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


@pytest.fixture(scope="session")
def pkg():
    return importlib.import_module(PKG)


@pytest.fixture(scope="session")
def sn():
    return importlib.import_module(PKG + ".synthnet")


@pytest.fixture(scope="session")
def abi():
    return importlib.import_module(PKG + ".abi")


@pytest.fixture(scope="session")
def wl():
    return importlib.import_module(PKG + ".workloads")


@pytest.fixture(scope="session")
def solver_mod():
    return importlib.import_module(PKG + ".solver")


@pytest.fixture(scope="session")
def orc():
    import oracle
    if not oracle.available():
        pytest.skip("oracle not built")
    return oracle
