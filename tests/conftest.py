"""Shared test configuration.

Markers:
  gpu   needs a CUDA device (B200); these are the parity tests proper and call
        the product through the C ABI of libolc.so.
Tests without the marker run on CPU: the oracle against the golden fixtures,
host-side logic, and that libolc.so loads and exports include/olc.h.
"""
from __future__ import annotations

import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")

# A checkout of the reference (yankokirill/Oncolytica), used only by the few
# CPU tests that read its example model: $OLC_REFERENCE, else a directory named
# "reference" beside this repository; those tests skip when neither exists.
REFERENCE = os.environ.get("OLC_REFERENCE") or os.path.join(os.path.dirname(REPO), "reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through libolc.so")


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def olc():
    from oncolytica_b200 import _lib

    return _lib.load()
