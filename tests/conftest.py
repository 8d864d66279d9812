"""Shared fixtures. Tests marked ``gpu`` need a CUDA device and the built library; the rest
run on the CPU (oracle pins, host logic, ABI exports, multi-process plumbing)."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "splatkit-ios_b200"))
sys.path.insert(0, str(ROOT))

from oracle import oracle as oracle_mod  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and libsplatkit_b200.so")


@pytest.fixture(scope="session")
def oracle():
    return oracle_mod.Oracle()


@pytest.fixture(scope="session")
def reference():
    if not oracle_mod.reference_available():
        pytest.skip("the reference C++ oracle (oracle/_ref) is not built")
    return oracle_mod.Reference()


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("a gpu-marked test ran without a CUDA device")
    return 0


def make_renderer(width, height, image_format=0):
    import splatkit_b200 as sk

    return sk.Renderer(width, height, image_format=image_format)
