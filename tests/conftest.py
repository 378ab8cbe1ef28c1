"""Shared test set-up: import paths, the `gpu` marker and library loaders."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PKG_DIR = os.path.join(ROOT, "slsf-rs_b200")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_package():
    """Import the package directory `slsf-rs_b200/` as module `slsf_rs_b200`."""
    if "slsf_rs_b200" in sys.modules:
        return sys.modules["slsf_rs_b200"]
    spec = importlib.util.spec_from_file_location(
        "slsf_rs_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["slsf_rs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def slsf():
    return load_package()
