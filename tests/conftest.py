"""Shared test setup: the `gpu` marker, the package loader and common fixtures."""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "oracle"))


def load_package():
    """Imports the package directory flame3d.jl_b200/ as the module `flame3d_b200`."""
    if "flame3d_b200" in sys.modules:
        return sys.modules["flame3d_b200"]
    pkg = ROOT / "flame3d.jl_b200"
    spec = importlib.util.spec_from_file_location("flame3d_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["flame3d_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def f3d():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    import oracle as o  # oracle/oracle.py
    o.load()
    return o


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
