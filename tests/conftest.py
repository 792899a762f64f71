import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def _load_package():
    if "cbm_b200" in sys.modules:
        return sys.modules["cbm_b200"]
    pkg = os.path.join(ROOT, "cellbasedmodels.jl_b200")
    spec = importlib.util.spec_from_file_location(
        "cbm_b200", os.path.join(pkg, "__init__.py"), submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cbm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


cbm = _load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libcbm_b200.so")


@pytest.fixture(scope="session")
def abi():
    return cbm._abi


@pytest.fixture(scope="session")
def gpu_lib():
    """The built product library; GPU tests fail loudly without it."""
    import torch
    assert torch.cuda.is_available(), "GPU test collected on a machine without CUDA"
    return cbm._abi.load_library()
