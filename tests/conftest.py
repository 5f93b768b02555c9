import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "residuum-solver_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def load_package():
    """Import residuum-solver_b200/ (a directory name that is not a Python identifier)."""
    name = "residuum_solver_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and librsd_cuda.so")


@pytest.fixture(scope="session")
def rsd():
    return load_package()


@pytest.fixture(scope="session")
def ctx(rsd):
    c = rsd.Context(0)
    yield c
    c.close()


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))
