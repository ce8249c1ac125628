"""Shared test setup.

Marker ``gpu``: the test needs a CUDA device (a B200). CPU-only runs use
``-m "not gpu"``. The CUDA library package lives in ``cup-cfd_b200/`` (a
directory name that is not a Python identifier), so it is loaded here by
path under the module name ``cupcfd_b200``; the test-only oracle is imported
from ``oracle/``.
"""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def load_cupcfd():
    name = "cupcfd_b200"
    if name in sys.modules:
        return sys.modules[name]
    path = os.path.join(ROOT, "cup-cfd_b200", "__init__.py")
    spec = importlib.util.spec_from_file_location(name, path, submodule_search_locations=[os.path.dirname(path)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def cg():
    return load_cupcfd()


@pytest.fixture(scope="session")
def gpu(cg):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    torch.cuda.init()
    return torch.device("cuda:0")
