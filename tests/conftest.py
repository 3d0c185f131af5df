"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "turbo-metrics_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, PKG_DIR)  # for `synth`


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def load_package():
    """Import the engine package (directory name `turbo-metrics_b200`) as `tmb`."""
    if "tmb" in sys.modules:
        return sys.modules["tmb"]
    spec = importlib.util.spec_from_file_location(
        "tmb", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["tmb"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def tmb():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    return o


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch
