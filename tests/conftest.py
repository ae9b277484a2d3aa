"""Shared test setup: paths, the `gpu` marker, oracle and library fixtures.

`-m "not gpu"` runs on a CPU-only machine: the oracle pinned against the reference's own
sources and golden vectors, the host logic, and the C-ABI library's exports. `-m gpu` runs the
parity tests of the CUDA path against the oracle (they need a CUDA device).
"""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
PKG_DIR = REPO / "gaussian-splat-renderer_b200"
for p in (REPO / "oracle", PKG_DIR, REPO / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (the parity tests of the CUDA path)")


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def port():
    from oracle import Oracle

    return Oracle("port")


@pytest.fixture(scope="session")
def ref():
    from oracle import Oracle, reference_available

    if not reference_available():
        pytest.skip("oracle/_ref (the reference compiled from its own sources) is not built here")
    return Oracle("reference")


@pytest.fixture(scope="session")
def gsr():
    import gsr_b200

    gsr_b200.load()
    return gsr_b200


@pytest.fixture(scope="session")
def gpu(gsr):
    if not cuda_available():
        pytest.fail("the gpu tests need a CUDA device")
    return gsr
