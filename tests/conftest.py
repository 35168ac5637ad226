"""Shared pytest configuration.

Markers: `gpu` tests need a CUDA device and the built product library;
everything else runs on CPU.  The product package directory has a hyphen in
its name, so it is loaded by path (see `load_product`).
"""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
PKG_DIR = os.path.join(ROOT, "paes-channelflow_b200")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def load_product():
    """Import paes-channelflow_b200/les_gpu.py (ctypes host layer) by path."""
    name = "les_gpu_host"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "les_gpu.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def product():
    return load_product()


@pytest.fixture(scope="session")
def gpu_lib(product):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return product.lib()
