"""Shared test setup.

Markers: `gpu` = needs a CUDA device (run on the B200 box with `-m gpu`).
The oracle libraries (oracle/_build, oracle/_ref) and the product library are
built on demand when missing, so `pytest -m "not gpu"` works from a clean tree.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_oracle():
    """Builds the oracle libraries when missing; oracle/Makefile builds the reference harness too
    when it finds the reference's sources (MSFEM_REFERENCE_DIR or its default)."""
    port = os.path.join(ROOT, "oracle", "_build", "libfemoracle.so")
    ref = os.path.join(ROOT, "oracle", "_ref", "libfemref.so")
    if not os.path.exists(port) or not os.path.exists(ref):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


def _ensure_lib():
    from multiscalefemsolver3d_b200 import build
    if not os.path.exists(build.LIB):
        build.build()


@pytest.fixture(scope="session")
def port():
    _ensure_oracle()
    import oracle
    return oracle.port()


@pytest.fixture(scope="session")
def ref():
    _ensure_oracle()
    import oracle
    if not oracle.ref_available():
        pytest.skip("reference harness (oracle/_ref/libfemref.so) not built on this machine")
    return oracle.ref()


@pytest.fixture(scope="session")
def lib():
    _ensure_lib()
    from multiscalefemsolver3d_b200 import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch.device("cuda:0")
