"""Test configuration: the `gpu` marker, in-tree builds, shared fixtures.

Tests marked ``gpu`` run the CUDA path on a B200 and compare it with the oracle; every
other test runs on the CPU (oracle pins against the reference, C-ABI exports, host-side
geometry, module logic, multi-process host logic over gloo).
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA kernels")


def _ensure_built():
    from imagingsuite_b200 import build

    build.build()
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)


_ensure_built()


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device for gpu tests; fails (does not skip) when no device is visible."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("gpu test selected but no CUDA device is visible")
    return torch.device("cuda", 0)


@pytest.fixture(scope="session")
def ref_lib():
    import oracle

    if not oracle.ref_available():
        pytest.skip("reference oracle not built (make -C oracle ref needs the reference tree)")
    return oracle.ref()
