"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on CPU.

The oracle (the reference renderer compiled from its own sources into
oracle/_ref by oracle/Makefile) is the checker; the GPU library under test is
marmel_trace_b200/libmtgpu.so.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

os.environ.setdefault("RAYTRACER_NO_PROGRESS", "1")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


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


@pytest.fixture(scope="session")
def mtlib():
    from marmel_trace_b200 import _capi, build

    build.build(verbose=False)
    return _capi.load()


@pytest.fixture(scope="session")
def oracle():
    from oracle import ref

    if not ref.available():
        pytest.skip("oracle library not built and reference sources absent")
    ref.load()
    return ref
