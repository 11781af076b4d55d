import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_product():
    """Import the product package directory ``raven.jl_b200`` as module ``raven_b200``."""
    if "raven_b200" in sys.modules:
        return sys.modules["raven_b200"]
    pkg_dir = os.path.join(ROOT, "raven.jl_b200")
    spec = importlib.util.spec_from_file_location(
        "raven_b200", os.path.join(pkg_dir, "__init__.py"), submodule_search_locations=[pkg_dir]
    )
    mod = importlib.util.module_from_spec(spec)
    sys.modules["raven_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def rb():
    return load_product()


@pytest.fixture(scope="session")
def cuda_ok():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
