"""Shared test setup: the `gpu` marker and loaders for the package and the oracle."""
import importlib.util
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PACKAGE_DIR = os.path.join(REPO, "fherma-polynomial-cuda_b200")
sys.path.insert(0, os.path.join(REPO, "tests"))
sys.path.insert(0, os.path.join(REPO, "tests", "golden"))


def _load(name, path, package_dir=None):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, path, submodule_search_locations=[package_dir] if package_dir else None)
    module = importlib.util.module_from_spec(spec)
    sys.modules[name] = module
    spec.loader.exec_module(module)
    return module


def load_package():
    """The B200 package (its directory name is not a Python identifier)."""
    return _load("fpc_b200", os.path.join(PACKAGE_DIR, "__init__.py"), PACKAGE_DIR)


def load_inputs():
    return _load("fpc_b200_inputs", os.path.join(PACKAGE_DIR, "inputs.py"))


def load_oracle():
    return _load("negacyclic_oracle", os.path.join(REPO, "oracle", "oracle.py"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")
    config.addinivalue_line("markers", "slow: full-size products (minutes)")


@pytest.fixture(scope="session")
def fpc():
    return load_package()


@pytest.fixture(scope="session")
def inputs():
    return load_inputs()


@pytest.fixture(scope="session")
def oracle():
    return load_oracle()
