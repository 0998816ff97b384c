"""Shared test setup: import paths, the `gpu` marker, built libraries."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "vapoursynth-bm3dcuda_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def engine_lib():
    """The in-tree engine library, built if missing (nvcc cross-compiles)."""
    so = os.path.join(PKG, "libbm3d_b200.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-s", "-C", PKG], check=True)
    from bm3dcuda import _lib
    return _lib.lib()


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build_port()
    return O


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test without a CUDA device: the engine has no CPU path")
    return torch
