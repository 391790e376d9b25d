"""Shared test set-up: paths, the `gpu` marker, and builds of the checkers.

`-m "not gpu"` tests run on any machine (the oracle, the host C++ surface,
the C ABI's symbol table); `-m gpu` tests need a CUDA device and compare the
CUDA path with the oracle through the C ABI.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _have_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _have_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def built():
    """Build the oracle (C restatement) and the product library if needed."""
    so = os.path.join(ROOT, "oracle", "libfluxos_oracle.so")
    src = os.path.join(ROOT, "oracle", "fluxos_oracle.c")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                       capture_output=True)
    from fluxos_cpp_b200 import build
    try:
        build.build()
    except RuntimeError:
        # nvcc is needed to build; tests that need the library will fail loudly.
        pass
    yield
