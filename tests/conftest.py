"""Shared pytest configuration: the ``gpu`` marker and the package loader.

Tests marked ``gpu`` need a CUDA device and the built libbass_b200.so; the
rest run on CPU (oracle against the reference's golden vectors, host logic,
C-ABI symbol checks)."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "bass-basis-adapative-sparse-simulations-_b200")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def load_pkg():
    """Import the package directory under the name ``bass_b200``."""
    if "bass_b200" in sys.modules:
        return sys.modules["bass_b200"]
    spec = importlib.util.spec_from_file_location("bass_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    m = importlib.util.module_from_spec(spec)
    sys.modules["bass_b200"] = m
    spec.loader.exec_module(m)
    return m


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built CUDA library")


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    oracle.build()
    return oracle
