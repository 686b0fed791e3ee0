"""Shared test setup.  GPU tests are marked ``gpu``; everything else runs on
a CPU-only machine."""
import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_package():
    name = "gevp_pdhgeqz_b200"
    if name in sys.modules:
        return sys.modules[name]
    path = os.path.join(ROOT, "gevp-pdhgeqz_b200", "__init__.py")
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def lapack():
    from oracle import lapack as L
    return L


EPS = np.finfo(np.float64).eps
