import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "ckks-train_b200")


def load_package():
    """Imports ckks-train_b200/ as the module ckks_train_b200."""
    if "ckks_train_b200" in sys.modules:
        return sys.modules["ckks_train_b200"]
    spec = importlib.util.spec_from_file_location(
        "ckks_train_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ckks_train_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


if os.path.join(ROOT, "oracle") not in sys.path:
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def ckg():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O
