"""Shared fixtures. GPU tests are marked ``gpu``; everything else runs on a CPU-only machine."""
from __future__ import annotations

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
    """Import the ``ops-blas_b200`` directory (not a valid identifier) as ``ops_blas_b200``."""
    name = "ops_blas_b200"
    if name in sys.modules:
        return sys.modules[name]
    path = os.path.join(ROOT, "ops-blas_b200", "__init__.py")
    spec = importlib.util.spec_from_file_location(name, path, submodule_search_locations=[os.path.dirname(path)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def ob():
    return load_package()


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without CUDA")
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def handle(ob, cuda):
    h = ob.Handle()
    yield h
    h.close()


def to_dev(a, device):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).to(device)


def to_host(t):
    return t.detach().cpu().numpy()
